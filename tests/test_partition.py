"""The C++ host partitioner (hif_partition.hpp) reproduces the reference's index data.

For every golden case the remaining-DOF mask is replayed phase by phase from the
reference's own eliminations; at each phase every cell's InteriorCellIndexData
must equal the reference's global / redundant / skeleton lists exactly, and every
face's SkelInteractionIndexData columns must equal the reference's face DOFs (its
rows are checked against the oracle restatement, which the reference pins).
CPU only.
"""
import numpy as np
import pytest

import goldens
import hifde3d_b200 as hb
from oracle import hif_oracle as ho

CASES = ["n8_unit", "n16_unit", "n16_unit_e3", "n16_rand", "n32_unit", "n32_rand"]


def initial_mask(NC):
    m = np.ones((NC, NC, NC), np.uint8)  # [k, j, i]
    m[0, :, :] = 0
    m[:, 0, :] = 0
    m[:, :, 0] = 0
    return m.ravel()


@pytest.mark.parametrize("name", CASES)
def test_partition_matches_reference(name):
    g = goldens.load(name)
    N, P, L = int(g["N"]), int(g["P"]), int(g["L"])
    NC = N + 1
    mask = initial_mask(NC)
    for lev in range(L):
        cpd = NC // ((1 << lev) * P)
        ref = list(goldens.blocks(g, lev, "schur"))
        assert len(ref) == cpd ** 3
        b = 0
        for ci in range(cpd):
            for cj in range(cpd):
                for ck in range(cpd):
                    gg, rr, ss = hb.partition_cell(N, P, lev, (ci, cj, ck), mask)
                    _, rg, rr_ref, rs_ref = ref[b]
                    np.testing.assert_array_equal(gg, rg)
                    np.testing.assert_array_equal(rr, rr_ref)
                    np.testing.assert_array_equal(ss, rs_ref)
                    b += 1
        for _, rg, rr_ref, _ in ref:
            mask[rg[rr_ref]] = 0
        if lev == L - 1:
            break
        refs = list(goldens.blocks(g, lev, "skel"))
        part = ho.Partition(N, P, mask.reshape(NC, NC, NC).transpose(2, 1, 0))
        f = 0
        for ci in range(cpd):
            for cj in range(cpd):
                for ck in range(cpd):
                    for face in (hb.TOP, hb.FRONT, hb.LEFT):
                        rows, cols = hb.partition_face(N, P, lev, (ci, cj, ck), face, mask)
                        orow, ocol = part.skel_interaction((ci, cj, ck), face, lev)
                        np.testing.assert_array_equal(rows, orow)
                        np.testing.assert_array_equal(cols, ocol)
                        if cols.size == 0:
                            continue
                        rface, rg, _, _ = refs[f]
                        assert rface == face
                        np.testing.assert_array_equal(cols, rg)
                        f += 1
        assert f == len(refs)
        for _, rg, rr_ref, _ in refs:
            mask[rg[rr_ref]] = 0
