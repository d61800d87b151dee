"""ComputeRowPtrs / ComputeColInds restated in the oracle, against the cases of
tests/unit_tests/solver/test_compute_row_ptrs.cpp and test_compute_col_inds.cpp."""
import numpy as np

from oracle.oracle_py import crs_build


def test_one_element_one_node():
    rp, ci = crs_build(6, 6, [6], [0], [[0]])
    assert list(rp) == [r * 6 for r in range(7)]
    assert list(ci) == list(range(6)) * 6


def test_one_element_two_nodes():
    rp, ci = crs_build(12, 12, [6, 6], [0, 6], [[0, 1]])
    assert list(rp) == [r * 12 for r in range(13)]
    assert list(ci) == list(range(12)) * 12


def test_two_elements_no_overlap():
    rp, ci = crs_build(24, 24, [6] * 4, [0, 6, 12, 18], [[0, 1], [2, 3]])
    assert list(rp) == [r * 12 for r in range(25)]
    for row in range(12):
        assert list(ci[row * 12:(row + 1) * 12]) == list(range(12))
    for row in range(12):
        assert list(ci[144 + row * 12:144 + (row + 1) * 12]) == [12 + c for c in range(12)]


def test_two_elements_overlap():
    rp, ci = crs_build(18, 18, [6] * 3, [0, 6, 12], [[0, 1], [1, 2]])
    assert list(rp[:7]) == [r * 12 for r in range(7)]
    assert list(rp[7:13]) == [72 + (r + 1) * 18 for r in range(6)]
    assert list(rp[13:19]) == [180 + (r + 1) * 12 for r in range(6)]
    for row in range(6):
        assert list(ci[row * 12:(row + 1) * 12]) == list(range(12))
        assert list(ci[72 + row * 18:72 + row * 18 + 12]) == list(range(12))
        assert list(ci[180 + row * 12:180 + (row + 1) * 12]) == [6 + c for c in range(12)]


def test_one_element_one_node_one_constraint():
    con = [{"base_active": 6, "target_active": 6, "base_table": [0, 1, 2, 3, 4, 5],
            "target_table": [6, 7, 8, 9, 10, 11], "row_range": [0, 6]}]
    rp, ci = crs_build(12, 18, [6, 6], [0, 6], [[0]], con)
    assert list(rp) == [r * 12 for r in range(19)]
    for row in range(6):
        e = rp[row]
        assert list(ci[e:e + 12]) == list(range(6)) + list(range(12, 18))
    for row in range(6, 12):
        e = rp[row]
        assert list(ci[e:e + 12]) == list(range(6, 12)) + list(range(12, 18))
    for row in range(12, 18):
        e = rp[row]
        assert list(ci[e:e + 12]) == list(range(12))


def test_unsorted_order_before_sort():
    """Constraint rows list target columns before base columns until sorted."""
    con = [{"base_active": 6, "target_active": 6, "base_table": [0, 1, 2, 3, 4, 5],
            "target_table": [6, 7, 8, 9, 10, 11], "row_range": [0, 6]}]
    rp, ci = crs_build(12, 18, [6, 6], [0, 6], [[0]], con, sort_rows=False)
    e = rp[12]
    assert list(ci[e:e + 12]) == list(range(6, 12)) + list(range(6))
