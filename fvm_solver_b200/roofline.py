"""Algorithmic (compulsory) bytes per kernel launch and per step, for roofline accounting.

Per kernel (``kernel_bytes``): every array a kernel must touch is counted once, 4 bytes per USED
element (8 per double); gathers of an array already counted are not counted again, and the padding
that rows carry for aligned vector accesses is not counted (``widths="stored"`` counts the stored
row widths instead, for comparison).  N cells, F facets, Fb boundary facets, d = dim, C = d + 2
components, K = d + 1 facets per cell, KG = d + 2 gradient slots.

Used elements per row (stored width in brackets, 2D / 3D):

* primitives, fluxes, boundary values  C              [4 / 8]
* limited gradients                    d C            [8 / 16]
* cell record   LSQ weights d KG, the KG - 1 neighbour columns, displacements K d, limiter eps
                                       18 / 32        [20 / 32]
* facet record  two side codes, 1/d, |S|, normal d, non-orthogonal vector d, two displacements
                d each                 12 / 16        [16 / 16]
* divergence record  +-1/vol K, facet ids K      6 / 8   [8 / 8]

k_cell      reads  cell records, primitives C N, boundary values C Fb; writes limited gradients d C N
k_face      reads  facet records, primitives C N, limited gradients d C N, boundary values C Fb,
                   boundary gradient rows 2 C Fb; writes fluxes C F
k_div_stage reads  divergence records, fluxes C F, state C N, stored increments C N each;
            writes primitives C N, stored increment C N (if kept), state C N (last stage)
k_bc        reads  cell primitives C Fb, tables (kind, b, ga, gb) 4 C Fb, lever arm d Fb,
                   characteristic data (2 + 2d) Fb, gradients of Neumann cells d C Fb;
            writes boundary values C Fb

Per step (``step_compulsory_bytes``): the traffic of a stage done in one pass, as the survey of
the reference path defines it -- per cell: state C + residual out C + LSQ weights d KG and columns
KG + neighbour map K + centroid->facet displacements K d + volume and limiter eps 2 + cell->facet
map and signs 2K + divergence operator 2K floats; per facet: normal d + non-orthogonal vector d +
projected distance 1 + facet->cell map 2 -- times 4 bytes, times the stages of the step.  In 3D
that is 256 B per cell + 36 B per facet (F = 2N: 328 B per cell-stage).
"""
from __future__ import annotations

from .tables import record_sizes, row_sizes


def used_record_sizes(dim: int) -> tuple:
    """(cell, facet, divergence) record elements that carry data."""
    K, KG = dim + 1, dim + 2
    cell = dim * KG + (KG - 1) + K * dim + 1        # compact record: weights, neighbour columns, disp, eps
    face = 4 + 4 * dim
    div = 2 * K
    return cell, face, div


def kernel_bytes(dim: int, N: int, F: int, Fb: int, kf: int | None = None, widths: str = "element") -> dict:
    C = dim + 2
    if widths == "element":
        R, G = C, dim * C
        CR, FR, DR = used_record_sizes(dim)
    elif widths == "stored":
        R, G = row_sizes(dim)
        CR, FR, DR = record_sizes(dim)
    else:
        raise ValueError(widths)
    w = 4
    cell = w * (CR * N + R * N + R * Fb + G * N)
    face = w * (FR * F + R * N + G * N + R * Fb + 2 * C * Fb + R * F)
    div_base = w * (DR * N + R * F + C * N + R * N)
    bc = w * (R * Fb + 4 * C * Fb + dim * Fb + (2 + 2 * dim) * Fb + G * Fb + R * Fb)
    return dict(cell=cell, face=face, div_base=div_base, bc=bc, row=w * N * C)


def div_stage_bytes(dim, N, F, Fb, stage_terms: list, kf=None, widths: str = "element") -> list:
    """Bytes of each k_div_stage launch of one step.

    ``stage_terms``: per stage (n_k_reads, store_k, final) -- increments read from memory, whether
    this stage's increment is stored, whether it writes the state.
    """
    kb = kernel_bytes(dim, N, F, Fb, kf, widths)
    return [kb["div_base"] + kb["row"] * (n_reads + int(store) + int(final)) for n_reads, store, final in stage_terms]


def step_compulsory_bytes(dim: int, N: int, F: int, stages: int) -> int:
    """One-pass compulsory bytes of a step of ``stages`` residual evaluations (see module doc)."""
    C, K, KG = dim + 2, dim + 1, dim + 2
    per_cell = C + C + dim * KG + KG + K + K * dim + 2 + 2 * K + 2 * K
    per_facet = dim + dim + 1 + 2
    return 4 * stages * (per_cell * N + per_facet * F)


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
