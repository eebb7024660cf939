"""The CIGAR regeneration's CPU restatement (oracle/cigar_oracle.py) on hand-derived cases
of scalar_banded_swa (banded_swa/scalar/implementation.rs:5-440) and infer_band_width
(region.rs:1277-1316), and the host mirror's band helper; no GPU needed."""
from oracle import cigar_oracle as C

MAT = [1 if t == q and t < 4 else (-1 if 4 in (t, q) else -4) for t in range(5) for q in range(5)]
P = {"mat": MAT, "o_del": 6, "e_del": 1, "o_ins": 6, "e_ins": 1, "zdrop": 100, "pen_clip3": 5}


def test_identical_sequences_one_match_run():
    s = [0, 1, 2, 3, 0, 1, 2, 3, 3, 2, 1, 0]
    out, cig, ra, qa = C.banded_swa(P, s, s, 10, 0)
    assert out == {"score": 12, "qle": 12, "tle": 12, "gtle": 12, "gscore": 12, "max_off": 0}
    assert cig == [("M", 12)] and ra == s and qa == s


def test_deletion_in_the_query():
    # target has two extra bases in the middle: 10 M, 2 D, 10 M once the flanks pay for the gap
    left = [0, 1, 2, 3, 3, 1, 0, 2, 1, 3]
    right = [2, 2, 1, 0, 3, 1, 2, 0, 0, 3]
    q = left + right
    t = left + [1, 1] + right
    out, cig, ra, qa = C.banded_swa(P, q, t, 10, 0)
    assert cig == [("M", 10), ("D", 2), ("M", 10)]
    assert out["score"] == 20 - 8 and out["qle"] == 20 and out["tle"] == 22
    assert ra == t and qa == q


def test_traceback_runs_to_the_matrix_edge():
    # the traceback does not stop where H falls to 0: it follows the stored codes to the
    # matrix edge, whose row 0 holds insertions, so extra leading query bases come out as an
    # I run rather than a 5' soft clip
    core = [0, 1, 2, 3, 3, 1, 0, 2, 1, 3, 2, 2, 1, 0]
    out, cig, ra, qa = C.banded_swa(P, [3, 3, 3] + core, core, 10, 0)
    assert cig == [("I", 3), ("M", 14)] and out["score"] == 14 and out["qle"] == 17
    assert ra == core and qa == [3, 3, 3] + core


def test_three_prime_clip_rule():
    core = [0, 1, 2, 3, 3, 1, 0, 2, 1, 3, 2, 2, 1, 0]
    # three mismatching tail bases: best gscore 5 <= 14 - pen_clip3 -> soft clip
    out, cig, _, _ = C.banded_swa(P, core + [3, 3, 3], core + [1, 1, 1], 10, 0)
    assert (out["score"], out["gscore"], cig) == (14, 5, [("M", 14), ("S", 3)])
    # one mismatching tail base: gscore 10 > 14 - 5 -> an M run to the query end (not merged
    # with the M before it, as in the reference)
    out, cig, _, _ = C.banded_swa(P, core + [3], core + [1], 10, 0)
    assert (out["gscore"], out["gtle"], cig) == (10, 15, [("M", 14), ("M", 1)])
    out, cig, _, _ = C.banded_swa({**P, "pen_clip3": 0}, core + [3], core + [1], 10, 0)
    assert cig == [("M", 14), ("S", 1)]


def test_empty_inputs():
    out, cig, ra, qa = C.banded_swa(P, [], [0, 1], 5, 0)
    assert out == {"score": 0, "qle": 0, "tle": 0, "gtle": 0, "gscore": 0, "max_off": 0} and cig == []


def test_band_width_known_values():
    # equal lengths and a near-perfect score: no band needed
    assert C.infer_band_width(100, 100, 100, 1, 6, 1, 6, 1, 100, 100) == 0
    # (min_len * a - score - o) / e + 2 = (100 - 80 - 6) + 2 = 16, above the length difference 10
    assert C.infer_band_width(100, 110, 80, 1, 6, 1, 6, 1, 100, 100) == 16
    # above the command-line band: the region's band caps it, and 4 * cmd_w caps that
    assert C.infer_band_width(300, 300, 20, 1, 6, 1, 6, 1, 50, 120) == 120
    assert C.infer_band_width(300, 300, 20, 1, 6, 1, 6, 1, 20, 500) == 80


def test_mirror_band_width_agrees(built):
    from ferrousalign_b200.cigar import infer_band_width
    import random
    rng = random.Random(3)
    for _ in range(2000):
        args = (rng.randint(0, 300), rng.randint(0, 300), rng.randint(-10, 300), rng.randint(1, 3),
                rng.randint(0, 10), rng.randint(0, 4), rng.randint(0, 10), rng.randint(0, 4),
                rng.randint(1, 150), rng.randint(1, 400))
        assert infer_band_width(*args) == C.infer_band_width(*args), args
