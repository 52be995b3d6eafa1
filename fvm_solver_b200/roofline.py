"""Algorithmic (compulsory) bytes per kernel launch, for roofline accounting.

Every array a kernel must touch is counted once (4 bytes per float / int32, 8 per double);
gathers of an array already counted are not counted again.  N cells, F facets, Fb boundary
facets, d = dim, C = d + 2 components, K = d + 1 facets per cell, KG = d + 2 gradient slots.

k_cell      reads  prims N C, G weights d KG N, G columns KG N, nb_slot N, disp K d N, eps N,
                   c2f K N, side N, boundary values Fb C
            writes facet values K N C, limited gradients N d C
k_face      reads  fcell 2F, fbc F, normals d F, fsize F, xorth d F, inv_d F, facet values 2F C,
                   limited gradients N d C, prims N C, boundary gradient rows 2 Fb C
            writes fluxes F C
k_div_stage reads  divergence weights + columns 2 K N, fluxes F C, state N C,
                   stored increments (one N C each)
            writes prims N C, stored increment N C (if kept), state N C (last stage)
k_bc        reads  cell prims Fb C, tables (kind, b, ga, gb) 4 Fb C, l d Fb, characteristic data
            writes boundary values 2 Fb C
"""
from __future__ import annotations


def kernel_bytes(dim: int, N: int, F: int, Fb: int, kf: int | None = None) -> dict:
    C, K, KG = dim + 2, dim + 1, dim + 2
    kf = kf or K
    w = 4
    cell = w * (N * C + dim * KG * N + KG * N + N + K * dim * N + N + K * N + N + Fb * C
                + K * N * C + N * dim * C)
    face = w * (2 * F + F + dim * F + F + dim * F + F + 2 * F * C + N * dim * C + N * C + 2 * Fb * C + F * C)
    div_base = w * (2 * kf * N + F * C + N * C + N * C)
    bc = w * (Fb * C + 4 * Fb * C + dim * Fb + 2 * Fb * C + 4 * Fb)
    return dict(cell=cell, face=face, div_base=div_base, bc=bc, row=w * N * C)


def div_stage_bytes(dim, N, F, Fb, stage_terms: list, kf=None) -> list:
    """Bytes of each k_div_stage launch of one step.

    ``stage_terms``: per stage (n_k_reads, store_k, final) -- increments read from memory, whether
    this stage's increment is stored, whether it writes the state.
    """
    kb = kernel_bytes(dim, N, F, Fb, kf)
    out = []
    for n_reads, store, final in stage_terms:
        out.append(kb["div_base"] + kb["row"] * (n_reads + int(store) + int(final)))
    return out


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
