"""The mate-rescue job collection's CPU restatement (oracle/mate_collect_oracle.py) on
hand-derived cases of collect_rescue_jobs_for_read_soa (mate_rescue.rs:1804-2045),
mem_infer_dir (:537-551) and bns_pos2rid / bns_fetch_seq (bntseq.rs:535-559, 700-739);
no GPU needed."""
import numpy as np

from oracle import mate_collect_oracle as M

OPT = {"pen_unpaired": 17, "max_matesw": 50, "min_seed_len": 19, "match_score": 1}
FR_ONLY = [{"low": 0, "high": 0, "failed": 1}, {"low": 200, "high": 600, "failed": 0},
           {"low": 0, "high": 0, "failed": 1}, {"low": 0, "high": 0, "failed": 1}]


def test_infer_dir_and_pos2rid():
    l_pac = 1000
    assert M.infer_dir(l_pac, 100, 400) == (0, 300)                 # same strand, mate to the right
    assert M.infer_dir(l_pac, 100, 2 * l_pac - 1 - 400) == (1, 300)  # other strand, projected right
    assert M.infer_dir(l_pac, 400, 100) == (3, 300)
    offs = [0, 300, 700]
    assert [M.pos2rid(offs, l_pac, p) for p in (0, 299, 300, 699, 700, 999, 1000)] == [0, 0, 1, 1, 2, 2, -1]


def _one_attempt(own, anchor, bounds=FR_ONLY):
    from ferrousalign_b200.collect import pack_reference
    rng = np.random.default_rng(5)
    ref = rng.integers(0, 4, 4000).astype(np.uint8)
    pac, l_pac = pack_reference(ref)
    chr_off, chr_len = [0, 2500], [2500, 1500]
    read = list(rng.integers(0, 5, 50))
    alns = own
    cand = {"read": 0, "aln_first": 0, "aln_count": len(own), "primary": 0, "anchor": anchor}
    return M.collect(OPT, bounds, pac, l_pac, chr_off, chr_len, [read], alns, [cand]), ref, read, l_pac


def test_fr_window_on_the_anchors_sequence():
    anchor = {"pos": 1000, "ref_id": 0, "is_rev": 0, "ref_len": 50, "score": 50}
    own = [{"pos": 100, "ref_id": 1, "is_rev": 0, "ref_len": 50, "score": 40}]   # elsewhere: no pair
    jobs, ref, read, l_pac = _one_attempt(own, anchor)
    assert len(jobs) == 1
    j = jobs[0]
    # FR (r = 1): reverse complement of the read; window [2 l_pac - 1 - (anchor + high) - ... ]:
    # is_rev, is_larger: rb = a + 200 - 50, re = a + 600, then mirrored by the midpoint's strand
    assert (j["orientation"], j["is_rev"], j["rid"]) == (1, 1, 0)
    assert (j["adj_rb"], j["adj_re"]) == (1000 + 200 - 50, 1000 + 600)
    assert j["query"] == [(3 - b if b < 4 else 4) for b in reversed(read)]
    assert j["target"] == list(ref[1150:1600])
    assert j["xtra"] == 0x40000 | 0x80000 | 0x10000 | 19


def test_paired_orientation_and_threshold_skip():
    anchor = {"pos": 1000, "ref_id": 0, "is_rev": 0, "ref_len": 50, "score": 50}
    # one of the read's alignments already pairs in FR (reverse strand, ending 399 bases right)
    mate_rb = 2 * 4000 - 1 - (1350 + 50 - 1)
    own = [{"pos": 1350, "ref_id": 0, "is_rev": 1, "ref_len": 50, "score": 40}]
    jobs, *_ = _one_attempt(own, anchor)
    assert jobs == [] and M.infer_dir(4000, 1000, mate_rb) == (1, 399)   # to its rightmost base
    # primary below best - pen_unpaired: no attempt (the alignments' best is 60, primary 30)
    own = [{"pos": 100, "ref_id": 1, "is_rev": 0, "ref_len": 50, "score": 30},
           {"pos": 300, "ref_id": 1, "is_rev": 0, "ref_len": 50, "score": 60}]
    jobs, *_ = _one_attempt(own, anchor)
    assert jobs == []


def test_window_cut_to_the_sequence_under_its_midpoint():
    own = [{"pos": 100, "ref_id": 1, "is_rev": 0, "ref_len": 50, "score": 40}]
    # FR window [2000 + 200 - 50, 2000 + 600) = [2150, 2600): midpoint 2375 in sequence 0,
    # which ends at 2500
    anchor = {"pos": 2000, "ref_id": 0, "is_rev": 0, "ref_len": 50, "score": 50}
    jobs, ref, _, _ = _one_attempt(own, anchor)
    assert [(j["adj_rb"], j["adj_re"]) for j in jobs] == [(2150, 2500)]
    assert jobs[0]["target"] == list(ref[2150:2500])
    # window [2350, 2800): its midpoint 2575 lies in sequence 1, not the anchor's: no job
    anchor = {"pos": 2200, "ref_id": 0, "is_rev": 0, "ref_len": 50, "score": 50}
    jobs, *_ = _one_attempt(own, anchor)
    assert jobs == []
