"""Host-side mirrors of the reference's operand structs for the Euler path.

Names and meaning follow src/StructsAndDictionaries.jl of DiplodocusTransport.jl:
``PhaseSpace`` mirrors PhaseSpaceStruct (:290) for the fields the step reads,
``BinaryMatrices`` mirrors BinaryMatricesStruct (:316), ``EmissionMatrices``
mirrors EmissionMatricesStruct (:329) and ``FluxMatrices`` mirrors
FluxMatricesStruct (:341).

Two equivalent forms of the binary operator are accepted:

* the reference layout ``M_Bin`` of size (n^2, n), column-major, where
  ``df_Bin[a] = Vol * sum_{j,k} M_Bin[j*n + a, k] f_j f_k``
  (src/SteppingMethods.jl:372-380, 0-based indices here), and
* the blocked form, a list of gain blocks ``G[a][b][c]`` (output species x
  input-1 species x input-2 species) and loss blocks ``L[a][c]`` such that
  ``df_Bin[a] = Vol * (sum_blk sum_{b,c} G[a][b][c] f_b f_c - f_a sum_blk sum_c L[a][c] f_c)``.

The blocked form is what BuildBinaryMatrices.jl:181-196 and :261-276 scatter
into M_Bin: a gain value ``val`` goes to M_Bin[(b-1)N+a, c] and M_Bin[(c-1)N+a, b]
as ``val/2`` each, a loss value to M_Bin[(a-1)N+a, c] and M_Bin[(c-1)N+a, a] as
``-val/2`` each. :func:`blocked_to_ref` performs exactly that scatter.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, List, Optional

import numpy as np


@dataclass
class PhaseSpace:
    """Momentum grid of each species and the space grid (single or multiple cells).

    State index of (cell, species s, px, py, pz), 0-based (GlobalToStateIndices.jl:22-25):
    ``cell * n_momentum + offset[s] + pz*px_num*py_num + py*px_num + px``.
    """

    name_list: List[str]
    px_num_list: List[int]
    py_num_list: List[int]
    pz_num_list: List[int]
    pxr_list: List[np.ndarray] = field(default_factory=list)
    pyr_list: List[np.ndarray] = field(default_factory=list)
    pzr_list: List[np.ndarray] = field(default_factory=list)
    mass_list: List[float] = field(default_factory=list)
    x_num: int = 1
    y_num: int = 1
    z_num: int = 1
    dt0: float = 1.0

    @property
    def species_sizes(self) -> List[int]:
        return [int(a * b * c) for a, b, c in zip(self.px_num_list, self.py_num_list, self.pz_num_list)]

    @property
    def momentum_species_offset(self) -> List[int]:
        """StructsAndDictionaries.jl:261-265, 0-based."""
        off, out = 0, []
        for n in self.species_sizes:
            out.append(off)
            off += n
        return out

    @property
    def n_momentum(self) -> int:
        return sum(self.species_sizes)

    @property
    def n_space(self) -> int:
        return self.x_num * self.y_num * self.z_num

    @property
    def n_state(self) -> int:
        return self.n_momentum * self.n_space

    def state_index(self, x: int, y: int, z: int, px: int, py: int, pz: int, species: int) -> int:
        """0-based GlobalIndices_To_StateIndex (GlobalToStateIndices.jl:7-27)."""
        pxn, pyn = self.px_num_list[species], self.py_num_list[species]
        off_space = x * self.y_num * self.z_num + y * self.z_num + z
        off_mom = pz * pxn * pyn + py * pxn + px
        return off_space * self.n_momentum + self.momentum_species_offset[species] + off_mom

    def species_slice(self, species: int, cell: int = 0) -> slice:
        """Location_Species_To_StateVector (GlobalToStateIndices.jl:35-63), 0-based slice."""
        start = cell * self.n_momentum + self.momentum_species_offset[species]
        return slice(start, start + self.species_sizes[species])


@dataclass
class GainBlock:
    """df[a] += sum_{b,c} G[a][b][c] f_b f_c; a in out_sp, b in in1_sp, c in in2_sp.

    ``G`` is a numpy array of shape (N_out, N_in1, N_in2) or a CUDA tensor of that shape.
    """

    out_sp: int
    in1_sp: int
    in2_sp: int
    G: Any


@dataclass
class LossBlock:
    """df[a] -= f_a * sum_c L[a][c] f_c; a in sp, c in other_sp. ``L``: (N_sp, N_other)."""

    sp: int
    other_sp: int
    L: Any


@dataclass
class EmiBlock:
    """A dense piece of M_Emi: rows [row0, row0+E.shape[0]), columns [col0, col0+E.shape[1])."""

    row0: int
    col0: int
    E: Any


@dataclass
class BinaryMatrices:
    M_Bin: Optional[np.ndarray] = None
    gains: List[GainBlock] = field(default_factory=list)
    losses: List[LossBlock] = field(default_factory=list)
    Domain: Optional[List[int]] = None

    @property
    def has_interactions(self) -> bool:
        """Binary_Interactions = !isempty(Binary_list) (SteppingStructs.jl:46)."""
        return self.M_Bin is not None or bool(self.gains) or bool(self.losses)


@dataclass
class EmissionMatrices:
    M_Emi: Optional[np.ndarray] = None
    blocks: List[EmiBlock] = field(default_factory=list)

    @property
    def has_interactions(self) -> bool:
        return self.M_Emi is not None or bool(self.blocks)


@dataclass
class FluxMatrices:
    """Ap_Flux must be diagonal (BuildFluxMatrices.jl:145-149); stored as a vector."""

    Ap_Flux: np.ndarray
    Am_Flux: np.ndarray
    X_Flux: Any  # scipy.sparse CSC, n x n
    P_Flux: Any  # scipy.sparse CSC, n x n
    Vol: np.ndarray  # one per space cell

    @property
    def F_Flux(self):
        """F = X + P (SteppingStructs.jl:60)."""
        return (self.X_Flux + self.P_Flux).tocsc()


def blocked_to_ref(ps: PhaseSpace, binm: BinaryMatrices) -> np.ndarray:
    """Scatter blocked gain/loss into the reference M_Bin layout (n^2, n), Fortran order.

    Follows BuildBinaryMatrices.jl:181-196 (gain) and :261-276 (loss), 0-based.
    """
    n = ps.n_momentum
    off = ps.momentum_species_offset
    M = np.zeros((n * n, n), dtype=np.float64, order="F")
    for g in binm.gains:
        G = np.asarray(g.G, dtype=np.float64)
        no, n1, n2 = G.shape
        a = off[g.out_sp] + np.arange(no)[:, None, None]
        b = off[g.in1_sp] + np.arange(n1)[None, :, None]
        c = off[g.in2_sp] + np.arange(n2)[None, None, :]
        a, b, c = np.broadcast_arrays(a, b, c)
        half = G / 2
        np.add.at(M, (b * n + a, c), half)
        np.add.at(M, (c * n + a, b), half)
    for l in binm.losses:
        L = np.asarray(l.L, dtype=np.float64)
        ns, no = L.shape
        a = off[l.sp] + np.arange(ns)[:, None]
        c = off[l.other_sp] + np.arange(no)[None, :]
        a, c = np.broadcast_arrays(a, c)
        half = L / 2
        np.add.at(M, (a * n + a, c), -half)
        np.add.at(M, (c * n + a, a), -half)
    return M


def emission_to_dense(ps: PhaseSpace, emim: EmissionMatrices) -> Optional[np.ndarray]:
    """Dense n x n M_Emi (Fortran order) from blocks, or the dense matrix itself."""
    if emim.M_Emi is not None:
        return np.asfortranarray(np.asarray(emim.M_Emi, dtype=np.float64))
    if not emim.blocks:
        return None
    n = ps.n_state
    M = np.zeros((n, n), dtype=np.float64, order="F")
    for b in emim.blocks:
        E = np.asarray(b.E, dtype=np.float64)
        M[b.row0:b.row0 + E.shape[0], b.col0:b.col0 + E.shape[1]] += E
    return M


def energy_weights(ps: PhaseSpace) -> np.ndarray:
    """Per-state cell-averaged energy used by the T^00 moment of one cell.

    DistributionMoments.jl:145 (m != 0) and :162 (m == 0); the weight depends on the
    p bin only and is repeated over the u and phi bins (p fastest).
    """
    out = []
    for s in range(len(ps.name_list)):
        pr = np.asarray(ps.pxr_list[s], dtype=np.float64)
        m = float(ps.mass_list[s])
        p0, p1 = pr[:-1], pr[1:]
        if m != 0.0:
            w = (p0 * np.sqrt(m * m + p0 * p0) - p1 * np.sqrt(m * m + p1 * p1)
                 + m * m * (np.arcsinh(p0 / m) - np.arcsinh(p1 / m))) / (2 * (p0 - p1))
        else:
            w = (p0 + p1) / 2
        reps = ps.py_num_list[s] * ps.pz_num_list[s]
        out.append(np.tile(w, reps))
    return np.concatenate(out)
