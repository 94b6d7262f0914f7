"""The x<->z swap matrices of the rotation M2L, derived from first principles
(taichi_collisional_b200/csrc/gen_swap_tables.py), against the reference's generated files
(multipole_rotation_matrix/rotate_order_{3..30}.txt, kernel_rotate.h:11-22)."""
import os
import re
import sys
from fractions import Fraction

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "taichi_collisional_b200", "csrc"))
import gen_swap_tables as g  # noqa: E402

import oracle  # noqa: E402

REF = oracle.reference_dir() or ""
MATS = g.derive(30)


def test_entries_are_dyadic_integers():
    for n in range(1, 31):
        g.integer_rows(MATS[n], n)  # asserts integrality of S * 2^(n-1)


def test_degree_one_and_two_hardcoded_rows():
    # kernel_rotate.h:11-22: arr[2]=old[3], arr[3]=old[2]; degree 2 with coeff 1/2
    S1 = MATS[1]
    assert S1[0] == [1, 0, 0] and S1[1] == [0, 0, 1] and S1[2] == [0, 1, 0]
    S2 = [[v * 2 for v in row] for row in MATS[2]]
    assert S2[0] == [0, 4, 0, 0, 0]
    assert S2[1] == [1, 0, 0, 0, 0]
    assert S2[2] == [0, 0, -1, 0, 1]
    assert S2[3] == [0, 0, 0, 2, 0]
    assert S2[4] == [0, 0, 3, 0, 1]


@pytest.mark.parametrize("n", range(1, 31))
def test_swap_is_an_involution(n):
    S = MATS[n]
    k = 2 * n + 1
    for i in range(k):
        for j in range(k):
            v = sum(S[i][q] * S[q][j] for q in range(k))
            assert v == (1 if i == j else 0)


def _parse(n):
    txt = open(os.path.join(REF, "multipole_rotation_matrix", "rotate_order_%d.txt" % n)).read()
    rows = {}
    for m in re.finditer(r"arr\[(\d+)\]=\((.*?)\)\*coeff", txt, re.S):
        body = m.group(2)
        rows[int(m.group(1))] = {int(j): int(c.replace(" ", "").replace("+", ""))
                                 for c, j in re.findall(r"([+-]\s*-?\d+)\s*\*\s*arrold\[(\d+)\]", body)}
    return rows


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "multipole_rotation_matrix")),
                    reason="reference tree not present")
@pytest.mark.parametrize("n", range(3, 31))
def test_matches_reference_files(n):
    rows = _parse(n)
    ir = g.integer_rows(MATS[n], n)
    for k in range(2 * n + 1):
        i = n * n + k
        mine = {n * n + j: v for j, v in enumerate(ir[k]) if v != 0}
        ref = rows.get(i, {})
        assert set(mine) == set(ref)
        for j in mine:
            if n <= 28:
                assert mine[j] == ref[j]
            else:  # literals above 2^53 are inexact in the reference (within one ulp)
                assert abs(mine[j] - ref[j]) <= 2 * abs(float(mine[j])) * 2.0 ** -52


def test_generated_header_is_current():
    hdr = os.path.join(HERE, "..", "taichi_collisional_b200", "csrc", "swap_tables.h")
    txt = open(hdr).read()
    pmax = int(re.search(r"#define TC_SWAP_PMAX (\d+)", txt).group(1))
    nnz = int(re.search(r"#define TC_SWAP_NNZ (\d+)", txt).group(1))
    expect = sum(1 for n in range(pmax + 1) for row in MATS[n] for v in row if v != Fraction(0))
    assert nnz == expect
