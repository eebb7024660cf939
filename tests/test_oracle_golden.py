"""The CPU oracle against the golden fixtures and known answers (no GPU).

The fixtures come from an independent pure-Python restatement
(tests/golden/make_golden.py); the known answers pin the reference's own unit test
(src/core/alignment/ksw_affine_gap.rs:1252-1277) and hand-derived cases.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import ksw_oracle as O

GOLD = Path(__file__).resolve().parent / "golden"


def enc(s):
    return np.array(["ACGT".index(c) if c in "ACGT" else 4 for c in s], np.uint8)


def kat_mat():
    m = np.full((5, 5), -1, np.int8)
    for i in range(4):
        m[i, i] = 1
    m[4, :] = 0
    m[:, 4] = 0
    return m.reshape(25)


def test_reference_unit_test_simple_match(built):
    # ksw_affine_gap.rs:1252-1277 asserts qle == 4, tle == 4 (and score > 10)
    r, tr = O.ksw_extend2(enc("ACGT"), enc("ACGT"), kat_mat(), 5, 1, 5, 1, 50, 0, 100, 10)
    assert r["qle"] == 4 and r["tle"] == 4 and r["score"] > 10
    # full hand-derived record: w clamps to max(0,(4-5)/1+1)->1; 4 matches on the diagonal
    assert tuple(r) == (14, 4, 4, 4, 14, 0)
    assert tr["w_eff"] == 1 and tr["rows"] == 4


def test_hand_derived_mismatch(built):
    # ACGT vs ACCT, h0=10: diagonal 11,12,11,12 -> max 12 at (1,1) then (3,3)? first strict max wins
    r, _ = O.ksw_extend2(enc("ACGT"), enc("ACCT"), kat_mat(), 5, 1, 5, 1, 50, 0, 100, 10)
    assert tuple(r) == (12, 2, 2, 4, 12, 0)


def test_h0_must_be_positive(built):
    with pytest.raises(ValueError):
        O.ksw_extend2(enc("ACGT"), enc("ACGT"), kat_mat(), 5, 1, 5, 1, 50, 0, 100, 0)


def test_empty_target(built):
    r, tr = O.ksw_extend2(enc("ACG"), enc(""), kat_mat(), 5, 1, 5, 1, 50, 0, 100, 7)
    assert tuple(r) == (7, 0, 0, 0, -1, 0) and tr["rows"] == 0


@pytest.mark.parametrize("case", json.loads((GOLD / "ext_cases.json").read_text()), ids=lambda c: c["name"])
def test_ext_golden(built, case):
    r, _ = O.ksw_extend2(case["query"], case["target"], case["mat"], case["o_del"], case["e_del"], case["o_ins"],
                         case["e_ins"], case["w"], case["end_bonus"], case["zdrop"], case["h0"])
    assert list(r) == case["expect"]


@pytest.mark.parametrize("case", json.loads((GOLD / "mate_cases.json").read_text()), ids=lambda c: c["name"])
def test_mate_golden(built, case):
    r = O.ksw_align2(case["query"], case["target"], case["mat"], case["o_del"], case["e_del"], case["o_ins"],
                     case["e_ins"], case["xtra"])
    assert list(r) == case["expect"]


def test_mate_reference_unit_tests(built):
    # ksw_affine_gap.rs:1393-1497 assert score > 0, te/qe >= 0, u8 score <= 255
    r = O.ksw_align2(enc("ACGTACGT"), enc("ACGTACGT"), kat_mat(), 5, 1, 5, 1, 0)
    assert r["score"] == 8 and r["te"] == 7 and r["qe"] == 7
    r = O.ksw_align2(enc("ACGTACGT"), enc("ACGTACGT"), kat_mat(), 5, 1, 5, 1, 0x80000)
    assert (r["tb"], r["qb"]) == (0, 0)
    r = O.ksw_align2(enc("ACGT"), enc("ACGT"), kat_mat(), 5, 1, 5, 1, 0x10000)
    assert 0 < r["score"] <= 255
