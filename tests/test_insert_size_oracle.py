"""The insert-size statistics' CPU restatement (oracle/insert_size_oracle.py) on
hand-derived cases of calculate_insert_size_stats (insert_size.rs:73-243); no GPU needed."""
from oracle import insert_size_oracle as S

L = 1_000_000


def fr(pos1, ins, read_len=100):
    # read 2 on the reverse strand ending ins - 1 bases after read 1's start
    return pos1, (L << 1) - 1 - (pos1 + ins - 1)


def test_orientation_and_distance():
    assert S.infer_orientation(L, 100, 400) == (0, 300)
    assert S.infer_orientation(L, *fr(100, 400)) == (1, 399)
    assert S.infer_orientation(L, 400, 100)[0] == 3


def test_uniform_fr_distribution():
    pairs = [fr(1000 + 7 * k, 301 + k % 100) for k in range(1000)]   # distances 300..399, ten of each
    st = S.stats(L, pairs)
    assert [s["failed"] for s in st] == [1, 0, 1, 1]
    fr_ = st[1]
    # sorted: ten copies of each of 300..399; p25 = s[250] = 325, p75 = s[750] = 375, iqr 50
    # 2-IQR bounds [225, 475] keep everything: mean 349.5, deviation sqrt((100^2 - 1) / 12)
    assert abs(fr_["avg"] - 349.5) < 1e-12
    assert abs(fr_["std"] - ((100 ** 2 - 1) / 12) ** 0.5) < 1e-9
    # proper pairs: 3 IQR -> [175, 525]; 4 sd (115.4) -> [188, 511]: the wider of each
    assert (fr_["low"], fr_["high"]) == (175, 525)


def test_too_few_and_ratio_failures():
    pairs = [fr(1000 + k, 300 + k % 7) for k in range(400)] + [(5000 + k, 5300 + k) for k in range(15)]
    st = S.stats(L, pairs)
    # FF has 15 pairs: enough for MIN_DIR_CNT, below 5% of FR's 400 -> failed
    assert st[0]["failed"] == 1 and st[1]["failed"] == 0
    assert S.stats(L, pairs[:9])[1]["failed"] == 1        # fewer than 10
