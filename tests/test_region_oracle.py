"""The region merge's CPU restatement (oracle/region_oracle.py) on hand-derived cases of
merge_scores_to_regions (src/pipelines/linear/region.rs:737-890), and the host mirror's
seed table; no GPU needed."""
import numpy as np

from oracle import region_oracle as R

OPT = {"a": 1, "pen_clip5": 5, "pen_clip3": 5, "w": 100}


def res(score, qle, tle, gtle, gscore):
    return {"score": score, "qle": qle, "tle": tle, "gtle": gtle, "gscore": gscore, "max_off": 0}


def seed(ref_pos, query_pos, ln, left=-1, right=-1):
    return {"ref_pos": ref_pos, "query_pos": query_pos, "len": ln, "left_job": left, "right_job": right}


def test_local_left_global_right():
    # left: gscore 40 <= score 45 - pen_clip5 -> local bounds from qle/tle, truesc = score
    # right: gscore 58 > 60 - pen_clip3 -> to the query end, re from gtle
    left = [res(45, 18, 19, 20, 40)]
    right = [res(60, 50, 52, 55, 58)]
    r = R.merge_chain(OPT, [seed(1000, 20, 30, 0, 0)], 101, left, right)
    assert (r["qb"], r["rb"], r["truesc"]) == (2, 981, 45)
    assert (r["qe"], r["re"]) == (101, 1000 + 30 + 55)
    assert r["score"] == 105 and r["seedlen0"] == 30 and r["seed"] == 0 and r["w"] == 100
    assert r["seedcov"] == 30


def test_global_left_local_right():
    left = [res(45, 18, 19, 20, 41)]          # 41 > 40: clipped to the query start
    right = [res(60, 50, 52, 55, 0)]          # gscore <= 0: local
    r = R.merge_chain(OPT, [seed(1000, 20, 30, 0, 0)], 101, left, right)
    assert (r["qb"], r["rb"], r["truesc"]) == (0, 980, 41)
    assert (r["qe"], r["re"]) == (20 + 30 + 50, 1000 + 30 + 52)


def test_seed_at_query_start_and_missing_jobs():
    # no left job and query_pos == 0: truesc = len * a; no right job: bounds stay the seed's
    r = R.merge_chain({**OPT, "a": 2}, [seed(500, 0, 25)], 80, [], [])
    assert (r["qb"], r["qe"], r["rb"], r["re"]) == (0, 25, 500, 525)
    assert r["score"] == 50 and r["truesc"] == 50
    # a left index past the results leaves everything (truesc falls back to the total)
    r = R.merge_chain(OPT, [seed(500, 10, 25, 3)], 80, [res(1, 1, 1, 1, 1)], [])
    assert (r["qb"], r["score"], r["truesc"]) == (10, 25, 25)
    # a query_pos > 0 seed without a left job keeps truesc 0 -> total
    r = R.merge_chain(OPT, [seed(500, 10, 25, -1, 0)], 80, [], [res(30, 20, 22, 22, 29)])
    assert r["score"] == 55 and r["truesc"] == 55 and r["qe"] == 80


def test_first_strict_maximum_and_coverage():
    left = [res(50, 10, 10, 10, 0), res(50, 5, 5, 5, 0)]
    seeds = [seed(2000, 40, 20, 0), seed(2030, 70, 10, 1), seed(1990, 30, 8)]
    r = R.merge_chain(OPT, seeds, 100, left, [])
    assert r["seed"] == 0 and r["score"] == 50       # tie at 50: the first one wins
    # region [30, 60) x [1990, 2020): seed 0 (40..60, 2000..2020) and seed 2 (30..38, 1990..1998)
    assert r["seedcov"] == 28
    r = R.merge_chain(OPT, seeds[::-1], 100, left, [])
    assert r["seed"] == 1   # reversed list: seed(2030..) is now first among the two 50s


def test_empty_chain_and_batch_driver():
    first = np.array([0, 0, 2], np.uint32)
    seeds = [seed(10, 0, 5), seed(40, 0, 9)]
    out = R.merge_regions(OPT, first, [50, 50], seeds, [], [])
    assert out[0]["seed"] == -1 and out[0]["w"] == 100
    assert out[1]["seed"] == 1 and out[1]["score"] == 9   # index into the whole seed array


def test_reference_positions_wrap_like_u64():
    r = R.merge_chain(OPT, [seed(3, 5, 4, 0)], 20, [res(9, 5, 10, 10, 0)], [])
    assert r["rb"] == (3 - 10) % (1 << 64)


def test_mirror_seed_table_uses_mapping_order(built):
    from ferrousalign_b200 import region as G
    first, seeds = G.chain_seed_table([[(100, 0, 10, None, 0), (200, 20, 10, 1, None)], []])
    assert list(first) == [0, 2, 2]
    assert list(seeds["ref_pos"]) == [200, 100]          # last seed of the chain first
    assert list(seeds["left_job"]) == [1, -1] and list(seeds["right_job"]) == [-1, 0]
    assert G.REGION_DT == R.REGION_DT and G.SEED_EXT_DT == R.SEED_EXT_DT
