"""The host partitioner against the oracle's restatement on arbitrary DOF masks (CPU).

The golden cases pin the partition to the reference for N <= 31 with the masks
the reference's own eliminations leave. The serving and bench sizes go further:
n = 48 and 96 use the clipped partition (cells of P * 2^l DOFs per side, the last
one per direction cut at N), and n = 64 and 128 (the bench's size) the reference
partition beyond the goldens. Cell and face index data depend only on the
remaining-DOF mask, so for random masks at every level both implementations must
produce identical lists:
global / redundant / skeleton positions of every cell (InteriorCellIndexData,
src/Factor.cpp:359-392) and rows / columns of every face
(SkelInteractionIndexData, src/Factor.cpp:645-755). Large levels are sampled,
always including the cells at the clipped boundary.
"""
import numpy as np
import pytest

import hifde3d_b200 as hb
from oracle import hif_oracle as ho


def random_mask(NC, keep, rng):
    m = (rng.random((NC, NC, NC)) < keep).astype(np.uint8)  # [k, j, i]
    m[0, :, :] = 0
    m[:, 0, :] = 0
    m[:, :, 0] = 0
    return m


def cells(cpd, limit, rng):
    allc = [(a, b, c) for a in range(cpd) for b in range(cpd) for c in range(cpd)]
    if len(allc) <= limit:
        return allc
    edge = [x for x in allc if cpd - 1 in x or 0 in x]
    pick = rng.choice(len(allc), limit, replace=False)
    return sorted(set(edge[: limit // 2]) | {allc[i] for i in pick})


@pytest.mark.parametrize("n,partition,limit", [(48, "clipped", 2000), (96, "clipped", 250),
                                               (64, "reference", 400), (128, "reference", 120)])
def test_partition_on_random_masks(n, partition, limit):
    N, P = n - 1, 4
    NC = N + 1
    rng = np.random.default_rng(n)
    L = ho.num_levels(N, P, partition)
    for lev in range(L):
        cpd = ho.cells_per_dir(N, P, lev, partition)
        m = random_mask(NC, 0.75 if lev == 0 else 0.4, rng)
        flat = m.ravel()
        part = ho.Partition(N, P, m.transpose(2, 1, 0))
        for cell in cells(cpd, limit, rng):
            g, r, s = hb.partition_cell(N, P, lev, cell, flat)
            og, orr, os_ = part.cell_index_data(cell, lev)
            np.testing.assert_array_equal(g, og)
            np.testing.assert_array_equal(r, orr)
            np.testing.assert_array_equal(s, os_)
            if lev == L - 1:
                continue
            for face in (hb.TOP, hb.FRONT, hb.LEFT):
                rows, cols = hb.partition_face(N, P, lev, cell, face, flat)
                orow, ocol = part.skel_interaction(cell, face, lev)
                np.testing.assert_array_equal(rows, orow)
                np.testing.assert_array_equal(cols, ocol)


def test_clipped_cells_cover_every_dof_once():
    """With the full mask, the clipped cells of level 0 at n = 48 hold every
    interior DOF exactly once as redundant or skeleton (no part of the domain is
    left out, unlike the reference's integer division for NC / P not a power of
    two, src/Factor.cpp:51-53)."""
    N, P = 47, 4
    NC = N + 1
    m = random_mask(NC, 1.1, np.random.default_rng(0))
    flat = m.ravel()
    cpd = ho.cells_per_dir(N, P, 0, "clipped")
    red = []
    skel = set()
    for a in range(cpd):
        for b in range(cpd):
            for c in range(cpd):
                g, r, s = hb.partition_cell(N, P, 0, (a, b, c), flat)
                red.extend(g[r].tolist())
                skel.update(g[s].tolist())
    assert len(red) == len(set(red))
    assert set(red).isdisjoint(skel)
    interior = set(np.flatnonzero(flat).tolist())
    # every DOF off the cell-boundary planes x, y, z = 4 q is redundant at level 0;
    # the rest lie on faces (skeleton) or on edges / corners (neither, yet)
    assert set(red) | skel <= interior
    on_planes = {d for d in interior
                 if (d % NC) % 4 == 0 or ((d // NC) % NC) % 4 == 0 or (d // (NC * NC)) % 4 == 0}
    assert set(red) == interior - on_planes
