"""Algorithmic (compulsory) bytes per kernel launch, for roofline accounting.

Every array a kernel must touch is counted once at its stored width (4 bytes per float / int32,
8 per double); gathers of an array already counted are not counted again.  N cells, F facets,
Fb boundary facets, d = dim, C = d + 2 components, K = d + 1 facets per cell; R = FVM_ROW (4 in
2D, 8 in 3D) floats per padded primitive / flux row, G = FVM_GROW (8 / 16) per limited-gradient
row, CR / FR / DR = cell / facet / divergence record widths (24 / 16 / 8 in 2D, 40 / 16 / 8 in 3D).

k_cell      reads  cell records CR N, primitives R N, boundary values R Fb
            writes limited gradients G N
k_face      reads  facet records FR F, primitives R N, limited gradients G N, boundary values R Fb,
                   boundary gradient rows 2 C Fb
            writes fluxes R F
k_div_stage reads  divergence records DR N, fluxes R F, state C N, stored increments C N each
            writes primitives R N, stored increment C N (if kept), state C N (last stage)
k_bc        reads  cell primitives R Fb, tables (kind, b, ga, gb) 4 C Fb, lever arm d Fb,
                   characteristic data (2 + 2d) Fb, gradients of Neumann cells G Fb
            writes boundary values R Fb
"""
from __future__ import annotations

from .tables import record_sizes, row_sizes


def kernel_bytes(dim: int, N: int, F: int, Fb: int, kf: int | None = None) -> dict:
    C = dim + 2
    R, G = row_sizes(dim)
    CR, FR, DR = record_sizes(dim)
    w = 4
    cell = w * (CR * N + R * N + R * Fb + G * N)
    face = w * (FR * F + R * N + G * N + R * Fb + 2 * C * Fb + R * F)
    div_base = w * (DR * N + R * F + C * N + R * N)
    bc = w * (R * Fb + 4 * C * Fb + dim * Fb + (2 + 2 * dim) * Fb + G * Fb + R * Fb)
    return dict(cell=cell, face=face, div_base=div_base, bc=bc, row=w * N * C)


def div_stage_bytes(dim, N, F, Fb, stage_terms: list, kf=None) -> list:
    """Bytes of each k_div_stage launch of one step.

    ``stage_terms``: per stage (n_k_reads, store_k, final) -- increments read from memory, whether
    this stage's increment is stored, whether it writes the state.
    """
    kb = kernel_bytes(dim, N, F, Fb, kf)
    return [kb["div_base"] + kb["row"] * (n_reads + int(store) + int(final)) for n_reads, store, final in stage_terms]


def tableau_terms(tab) -> list:
    """(k reads, store_k, final) per stage for an fvm_tableau_t (mirrors stage_args in residual.cu)."""
    S = tab.stages
    terms = []
    for s in range(S):
        if s < S - 1:
            reads = sum(1 for j in range(s) if tab.a[s + 1][j] != 0.0)
            needed = tab.b[s] != 0.0 or (tab.adaptive and tab.b2[s] != 0.0)
            needed = needed or any(tab.a[i][s] != 0.0 for i in range(s + 2, S))
            terms.append((reads, bool(needed), False))
        else:
            reads = sum(1 for j in range(S - 1) if tab.b[j] != 0.0)
            if tab.adaptive:
                reads += sum(1 for j in range(S - 1) if tab.b2[j] != 0.0 and tab.b[j] == 0.0)
            terms.append((reads, False, True))
    return terms
