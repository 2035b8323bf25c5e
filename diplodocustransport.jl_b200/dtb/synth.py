"""Seeded synthetic workloads for the Euler path (no collision data files are needed).

Every config is built from a seed; the recipe follows the workload description of each
config (grid, flux stencil, log-uniform gain/loss/emission values, log-normal initial f):

* flux F: upwind finite-volume stencil coupling nearest neighbours in p and u (closed
  boundaries, <= 5 nonzeros per row). Each interior face carries a seeded velocity
  U[-1, 1]; the upwind cell loses it and the downwind cell gains it, so columns sum to zero
  (number conserving) and the diagonal is non-negative. The whole matrix is rescaled so
  that dt * spectral_radius(diag(invAp) F) = 0.4, which keeps the explicit step positive.
* gain G, loss L, emission E: entries 10**U[lo, hi]; each block is multiplied by a
  recorded scale ``kappa`` chosen so that, at f normalised to unit number per species,
  the block moves a fixed fraction of a species' number per step (gain 0.5%, loss 1%,
  emission 0.5%). Loss outweighs gain, so runs do not blow up over thousands of steps.
* f0: log-normal in p (ln p ~ N(mu, sigma)), integrated over each p bin, isotropic in u,
  normalised to unit number per species.

Scales are returned in ``meta`` so a run can be reproduced exactly.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .structs import (BinaryMatrices, EmiBlock, EmissionMatrices, FluxMatrices, GainBlock,
                      LossBlock, PhaseSpace)

RATE_GAIN = 0.005
RATE_LOSS = 0.01
RATE_EMI = 0.005
CFL_TARGET = 0.4


@dataclass
class Workload:
    ps: PhaseSpace
    binm: BinaryMatrices
    emim: EmissionMatrices
    fluxm: FluxMatrices
    f0: np.ndarray  # (n,) or (batch, n)
    inj: np.ndarray  # (n,)
    dt: Any  # float or (batch,) array
    n_steps: int
    meta: Dict[str, Any] = field(default_factory=dict)


def log_uniform_mean(lo: float, hi: float) -> float:
    """Mean of 10**U[lo, hi]."""
    return (10.0 ** hi - 10.0 ** lo) / ((hi - lo) * math.log(10.0))


def phase_space(names: List[str], p_num: int, p_lo: float, p_hi: float, u_num: int,
                masses: List[float], dt0: float = 1.0, x_num: int = 1) -> PhaseSpace:
    """Log-spaced p bounds over [p_lo, p_hi], uniform u = cos(theta) on [-1, 1], one phi bin
    on [0, 2] (phi/pi, Constants.jl:43-44)."""
    ns = len(names)
    pr = np.logspace(math.log10(p_lo), math.log10(p_hi), p_num + 1)
    ur = np.linspace(-1.0, 1.0, u_num + 1)
    hr = np.array([0.0, 2.0])
    return PhaseSpace(name_list=list(names), px_num_list=[p_num] * ns, py_num_list=[u_num] * ns,
                      pz_num_list=[1] * ns, pxr_list=[pr.copy() for _ in range(ns)],
                      pyr_list=[ur.copy() for _ in range(ns)], pzr_list=[hr.copy() for _ in range(ns)],
                      mass_list=list(masses), x_num=x_num, dt0=dt0)


def upwind_flux(ps: PhaseSpace, rng: np.random.Generator, dt: float,
                cfl: float = CFL_TARGET) -> FluxMatrices:
    """Nearest-neighbour upwind stencil in p and u for every species and cell."""
    n = ps.n_state
    rows, cols, vals = [], [], []
    for cell in range(ps.n_space):
        for s in range(len(ps.name_list)):
            pn, un = ps.px_num_list[s], ps.py_num_list[s]
            base = cell * ps.n_momentum + ps.momentum_species_offset[s]
            # faces in p: between (p, u) and (p+1, u); faces in u: between (p, u) and (p, u+1)
            for axis, (na, nb, stride) in enumerate(((pn - 1, un, 1), (pn, un - 1, pn))):
                v = rng.uniform(-1.0, 1.0, size=(nb, na))
                for j in range(nb):
                    for i in range(na):
                        lo = base + j * pn + i
                        hi = lo + stride
                        w = v[j, i]
                        src, dst = (lo, hi) if w > 0 else (hi, lo)
                        aw = abs(w)
                        rows += [src, dst]
                        cols += [src, src]
                        vals += [aw, -aw]
    F = sp.csc_matrix((vals, (rows, cols)), shape=(n, n))
    F.sum_duplicates()
    invAp = np.ones(n)
    if F.nnz:
        if n <= 256:
            rho = float(np.max(np.abs(np.linalg.eigvals(F.toarray()))))
        else:
            rho = abs(spla.eigs(F.astype(np.float64), k=1, which="LM", return_eigenvectors=False,
                                tol=1e-10, maxiter=100000)[0])
        F = F * (cfl / (dt * rho))
    F = F.tocsc()
    F.sort_indices()
    X = sp.csc_matrix((n, n))
    return FluxMatrices(Ap_Flux=1.0 / invAp, Am_Flux=-1.0 / invAp, X_Flux=X, P_Flux=F,
                        Vol=np.ones(ps.n_space))


def space_flux(ps: PhaseSpace, rng: np.random.Generator, dt: float, cfl: float = 0.2):
    """Upwind flux of every momentum state between neighbouring space cells (closed ends): a
    seeded velocity U[-1, 1] per (face, state); columns sum to zero. Scaled so that
    dt * spectral_radius = cfl."""
    n, nm = ps.n_state, ps.n_momentum
    rows, cols, vals = [], [], []
    for cell in range(ps.n_space - 1):
        v = rng.uniform(-1.0, 1.0, size=nm)
        for m in range(nm):
            lo, hi = cell * nm + m, (cell + 1) * nm + m
            src, dst = (lo, hi) if v[m] > 0 else (hi, lo)
            aw = abs(v[m])
            rows += [src, dst]
            cols += [src, src]
            vals += [aw, -aw]
    X = sp.csc_matrix((vals, (rows, cols)), shape=(n, n))
    X.sum_duplicates()
    if X.nnz:
        rho = float(np.max(np.abs(np.linalg.eigvals(X.toarray())))) if n <= 512 else abs(
            spla.eigs(X, k=1, which="LM", return_eigenvectors=False)[0])
        X = X * (cfl / (dt * rho))
    X = X.tocsc()
    X.sort_indices()
    return X


def lognormal_f0(ps: PhaseSpace, mu: List[float], sigma: float = 1.0) -> np.ndarray:
    """Cell-integrated log-normal p spectrum, isotropic in u, unit number per species."""
    f = np.zeros(ps.n_state)
    for cell in range(ps.n_space):
        for s in range(len(ps.name_list)):
            pr = ps.pxr_list[s]
            z = (np.log(pr) - mu[s]) / sigma
            cdf = 0.5 * (1.0 + np.array([math.erf(x / math.sqrt(2.0)) for x in z]))
            w = np.diff(cdf)
            w = w / w.sum()
            un = ps.py_num_list[s] * ps.pz_num_list[s]
            block = np.tile(w / un, un)
            sl = ps.species_slice(s, cell)
            f[sl] = block
    return f


def _log_uniform(rng: np.random.Generator, shape, lo: float, hi: float) -> np.ndarray:
    return 10.0 ** rng.uniform(lo, hi, size=shape)


def gain_kappa(lo: float, hi: float, n_out: int, dt: float) -> float:
    return RATE_GAIN / (dt * log_uniform_mean(lo, hi) * n_out)


def loss_kappa(lo: float, hi: float, dt: float) -> float:
    return RATE_LOSS / (dt * log_uniform_mean(lo, hi))


def emi_kappa(lo: float, hi: float, n_rows: int, dt: float) -> float:
    return RATE_EMI / (dt * log_uniform_mean(lo, hi) * n_rows)


def two_species(p_num: int, p_lo: float, p_hi: float, u_num: int, seed: int, dt: float = 1.0,
                g_range=(-6.0, 0.0), with_emission: bool = True, gain_on_device: bool = False,
                gain_dtype=None, n_space: int = 1, device: str = "cuda",
                gain_rows: Optional[int] = None) -> Workload:
    """Electron + photon workload with an e + gamma -> e + gamma binary interaction.

    ``gain_rows`` keeps only the first rows of each gain block (host timing samples)."""
    ps = phase_space(["Ele", "Pho"], p_num, p_lo, p_hi, u_num, [1.0, 0.0], dt0=1.0, x_num=n_space)
    rng = np.random.default_rng(seed)
    fluxm = upwind_flux(ps, rng, dt)
    ns = ps.species_sizes[0]
    lo, hi = g_range
    kg = gain_kappa(lo, hi, ns, dt)
    gains = []
    for out in (0, 1):
        if gain_on_device:
            G = device_log_uniform((ns, ns, ns), lo, hi, kg, seed * 1000 + 17 + out,
                                   gain_dtype, device)
        else:
            G = _log_uniform(rng, (gain_rows or ns, ns, ns), lo, hi) * kg
        gains.append(GainBlock(out, 0, 1, G))
    kl = loss_kappa(lo, hi, dt)
    losses = [LossBlock(0, 1, _log_uniform(rng, (ns, ns), lo, hi) * kl),
              LossBlock(1, 0, _log_uniform(rng, (ns, ns), lo, hi) * kl)]
    emim = EmissionMatrices()
    ke = emi_kappa(lo, hi, ns, dt)
    if with_emission:
        emim.blocks.append(EmiBlock(row0=ps.momentum_species_offset[1], col0=0,
                                    E=_log_uniform(rng, (ns, ns), lo, hi) * ke))
    f0 = lognormal_f0(ps, [0.0, 0.0], 1.0)
    return Workload(ps=ps, binm=BinaryMatrices(gains=gains, losses=losses), emim=emim,
                    fluxm=fluxm, f0=f0, inj=np.zeros(ps.n_state), dt=dt, n_steps=0,
                    meta=dict(seed=seed, kappa_gain=kg, kappa_loss=kl, kappa_emi=ke,
                              g_range=g_range))


def uneven_two_species(p_e: int, u_e: int, p_g: int, u_g: int, seed: int, batch: Optional[int] = None,
                       dt_max: float = 1.0, g_range=(-6.0, 0.0), p_lo: float = 1e-2, p_hi: float = 1e2) -> Workload:
    """Electron + photon workload on grids of different sizes (p_e x u_e electron states, p_g x u_g
    photon states; the same p range): gain blocks n_out x n_e x n_g, loss blocks of both sides,
    photon emission from electrons. With ``batch``, per-instance f0 and dt as batched_two_species."""
    pe = np.logspace(math.log10(p_lo), math.log10(p_hi), p_e + 1)
    pg = np.logspace(math.log10(p_lo), math.log10(p_hi), p_g + 1)
    hr = np.array([0.0, 2.0])
    ps = PhaseSpace(name_list=["Ele", "Pho"], px_num_list=[p_e, p_g], py_num_list=[u_e, u_g], pz_num_list=[1, 1],
                    pxr_list=[pe, pg], pyr_list=[np.linspace(-1.0, 1.0, u_e + 1), np.linspace(-1.0, 1.0, u_g + 1)],
                    pzr_list=[hr.copy(), hr.copy()], mass_list=[1.0, 0.0], x_num=1, dt0=1.0)
    rng = np.random.default_rng(seed)
    fluxm = upwind_flux(ps, rng, dt_max)
    ne, ng = ps.species_sizes
    lo, hi = g_range
    gains = [GainBlock(out, 0, 1, _log_uniform(rng, (n_out, ne, ng), lo, hi) * gain_kappa(lo, hi, n_out, dt_max))
             for out, n_out in ((0, ne), (1, ng))]
    kl = loss_kappa(lo, hi, dt_max)
    losses = [LossBlock(0, 1, _log_uniform(rng, (ne, ng), lo, hi) * kl),
              LossBlock(1, 0, _log_uniform(rng, (ng, ne), lo, hi) * kl)]
    emim = EmissionMatrices()
    emim.blocks.append(EmiBlock(row0=ps.momentum_species_offset[1], col0=0,
                                E=_log_uniform(rng, (ng, ne), lo, hi) * emi_kappa(lo, hi, ng, dt_max)))
    w = Workload(ps=ps, binm=BinaryMatrices(gains=gains, losses=losses), emim=emim, fluxm=fluxm,
                 f0=lognormal_f0(ps, [0.0, 0.0], 1.0), inj=np.zeros(ps.n_state), dt=dt_max, n_steps=0,
                 meta=dict(seed=seed))
    if batch is not None:
        r2 = np.random.default_rng(seed + 7)
        mus = r2.uniform(-1.0, 1.0, size=batch)
        w.f0 = np.stack([lognormal_f0(ps, [mu, mu], 1.0) for mu in mus])
        w.dt = r2.uniform(0.5, 1.0, size=batch) * dt_max
    return w


def device_log_uniform(shape, lo: float, hi: float, kappa: float, seed: int, dtype=None,
                       device: str = "cuda"):
    """10**U[lo, hi] * kappa generated on a CUDA device with a seeded torch generator."""
    import torch
    dtype = dtype or torch.float32
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.empty(shape, dtype=dtype, device=device)
    flat = out.view(-1)
    chunk = 1 << 27
    for s in range(0, flat.numel(), chunk):
        e = min(flat.numel(), s + chunk)
        u = torch.rand(e - s, generator=g, device=device, dtype=torch.float32)
        flat[s:e] = (torch.pow(10.0, lo + (hi - lo) * u) * kappa).to(dtype)
    return out


def config0(seed: int = 0) -> Workload:
    """Plain method, FP64: 16 p bins over 1e-2..1e2 x 8 u bins, 2 species, 1000 steps."""
    w = two_species(16, 1e-2, 1e2, 8, seed)
    w.n_steps = 1000
    return w


def config1(seed: int = 1, gain_on_device: bool = True, device: str = "cuda",
            gain_rows: Optional[int] = None) -> Workload:
    """Plain single instance: 64 p bins over 1e-3..1e3 x 16 u bins (1024 states per species),
    FP32 gain tensor 1024 x 1,048,576 per output species, 2000 steps."""
    w = two_species(64, 1e-3, 1e3, 16, seed, gain_on_device=gain_on_device, device=device,
                    gain_rows=gain_rows)
    w.n_steps = 2000
    return w


def small(p_num: int = 4, u_num: int = 2, seed: int = 0, dt: float = 1.0, n_space: int = 1,
          with_emission: bool = True, randomize_vectors: bool = False) -> Workload:
    """Small two-species workload for parity tests; optionally random invAp, Vol and inj."""
    w = two_species(p_num, 1e-2, 1e2, u_num, seed, dt=dt, with_emission=with_emission,
                    n_space=n_space)
    if randomize_vectors:
        rng = np.random.default_rng(seed + 99)
        n = w.ps.n_state
        w.fluxm.Ap_Flux = rng.uniform(0.8, 1.25, n)
        w.fluxm.Am_Flux = -w.fluxm.Ap_Flux
        w.fluxm.Vol = rng.uniform(0.5, 1.5, w.ps.n_space)
        w.inj = rng.uniform(0.0, 1e-4, n)
    w.n_steps = 20
    return w


def batched_two_species(p_num: int, p_lo: float, p_hi: float, u_num: int, batch: int, seed: int,
                        dt_max: float = 1.0, g_range=(-6.0, 0.0), gain_on_device: bool = False,
                        device: str = "cuda", with_emission: bool = True) -> Workload:
    """Shared e + gamma operators and `batch` instances: f0 log-normal in p with mean log p drawn
    from U[-1, 1] per instance, dt drawn from U[0.5, 1] * dt_max per instance."""
    w = two_species(p_num, p_lo, p_hi, u_num, seed, dt=dt_max, g_range=g_range, gain_on_device=gain_on_device,
                    device=device, with_emission=with_emission)
    rng = np.random.default_rng(seed + 7)
    mus = rng.uniform(-1.0, 1.0, size=batch)
    w.f0 = np.stack([lognormal_f0(w.ps, [mu, mu], 1.0) for mu in mus])
    w.dt = rng.uniform(0.5, 1.0, size=batch) * dt_max
    w.meta["mu"] = mus
    return w


def config2(seed: int = 2, gain_on_device: bool = True, device: str = "cuda") -> Workload:
    """Batching: 256 instances on 32 log p bins over 1e-2..1e2 x 8 u bins (256 states per
    species), one shared G (2 x 256 x 65,536), 10,000 steps."""
    w = batched_two_species(32, 1e-2, 1e2, 8, 256, seed, gain_on_device=gain_on_device, device=device)
    w.n_steps = 10000
    return w


def synchrotron_like(ps: PhaseSpace, emitter: int, photon: int, B: float, kappa: float) -> np.ndarray:
    """Photon rows x emitter columns: kappa * B^2 * x^(1/3) exp(-x), x = eps_gamma / eps_c,
    eps_c = 1.5 B gamma^2 (gamma from the emitter's p-bin mean, mass 1), isotropic in u."""
    pe = np.sqrt(ps.pxr_list[emitter][:-1] * ps.pxr_list[emitter][1:])
    pg = np.sqrt(ps.pxr_list[photon][:-1] * ps.pxr_list[photon][1:])
    gam = np.sqrt(1.0 + pe * pe)
    x = pg[:, None] / (1.5 * B * gam[None, :] ** 2)
    k = kappa * B * B * np.cbrt(x) * np.exp(-np.minimum(x, 700.0))  # (p_gamma, p_e)
    ug, ue = ps.py_num_list[photon], ps.py_num_list[emitter]
    E = np.zeros((ps.species_sizes[photon], ps.species_sizes[emitter]))
    pn_g, pn_e = ps.px_num_list[photon], ps.px_num_list[emitter]
    for jg in range(ug):
        for je in range(ue):
            E[jg * pn_g:(jg + 1) * pn_g, je * pn_e:(je + 1) * pn_e] = k / ug
    return E


def three_species(p_num: int, p_lo: float, p_hi: float, u_num: int, batch: int, seed: int,
                  gain_on_device: bool = False, device: str = "cuda", g_range=(-8.0, 0.0)) -> Workload:
    """Electrons, positrons, photons with e- + gamma and e+ + gamma Compton-like gain/loss and
    gamma + gamma -> e+ e- pair gain/loss; synchrotron-like emission of e-/e+ into photons from a
    uniform B of seeded magnitude; `batch` instances with log-normal f0 and dt in [0.5, 1]."""
    ps = phase_space(["Ele", "Pos", "Pho"], p_num, p_lo, p_hi, u_num, [1.0, 1.0, 0.0])
    rng = np.random.default_rng(seed)
    fluxm = upwind_flux(ps, rng, 1.0)
    ns = ps.species_sizes[0]
    lo, hi = g_range
    kg = gain_kappa(lo, hi, ns, 1.0)
    blocks = [(0, 0, 2), (2, 0, 2), (1, 1, 2), (2, 1, 2), (0, 2, 2), (1, 2, 2)]
    gains = []
    for k, (o, a, b) in enumerate(blocks):
        if gain_on_device:
            G = device_log_uniform((ns, ns, ns), lo, hi, kg, seed * 1000 + 31 + k, None, device)
        else:
            G = _log_uniform(rng, (ns, ns, ns), lo, hi) * kg
        gains.append(GainBlock(o, a, b, G))
    kl = loss_kappa(lo, hi, 1.0)
    losses = [LossBlock(s_, o, _log_uniform(rng, (ns, ns), lo, hi) * kl)
              for s_, o in ((0, 2), (2, 0), (1, 2), (2, 1), (2, 2))]
    Bmag = float(10.0 ** rng.uniform(-1.0, 1.0))
    emim = EmissionMatrices()
    for em in (0, 1):
        E = synchrotron_like(ps, em, 2, Bmag, 1.0)
        E *= RATE_EMI / max(E.sum(axis=0).max(), 1e-300)  # largest column moves 0.5% per step
        emim.blocks.append(EmiBlock(row0=ps.momentum_species_offset[2], col0=ps.momentum_species_offset[em], E=E))
    rng2 = np.random.default_rng(seed + 7)
    mus = rng2.uniform(-1.0, 1.0, size=batch)
    f0 = np.stack([lognormal_f0(ps, [mu, mu, mu], 1.0) for mu in mus])
    dts = rng2.uniform(0.5, 1.0, size=batch)
    return Workload(ps=ps, binm=BinaryMatrices(gains=gains, losses=losses), emim=emim, fluxm=fluxm, f0=f0,
                    inj=np.zeros(ps.n_state), dt=dts, n_steps=0,
                    meta=dict(seed=seed, kappa_gain=kg, kappa_loss=kl, B=Bmag, mu=mus))


def config3(seed: int = 3, batch: int = 64, gain_on_device: bool = True, device: str = "cuda") -> Workload:
    """Mixed precision, three interactions: electrons, positrons, photons on 48 log p bins over
    1e-3..1e3 x 12 u bins (576 states per species), each gain tensor 576 x 331,776 with values
    log-uniform over 1e-8..1; 64 instances, 5000 steps."""
    w = three_species(48, 1e-3, 1e3, 12, batch, seed, gain_on_device=gain_on_device, device=device)
    w.n_steps = 5000
    return w
