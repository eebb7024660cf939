"""The job collection's CPU restatement (oracle/collect_oracle.py) on hand-derived cases of
collect_extension_jobs_batch_soa (collect_soa.rs:28-230), cal_max_gap
(chaining.rs:1108-1116) and the packed-reference reads (bntseq.rs:451-575); no GPU needed."""
import numpy as np

from oracle import collect_oracle as C

OPT = {"a": 1, "o_del": 6, "e_del": 1, "o_ins": 6, "e_ins": 1, "w": 100}


def test_cal_max_gap_known_values():
    assert C.cal_max_gap(OPT, 100) == 95          # (100 - 6) / 1 + 1
    assert C.cal_max_gap(OPT, 300) == 200         # capped at 2w
    assert C.cal_max_gap(OPT, 0) == 1             # (0 - 6) / 1 + 1 = -5 -> at least 1
    assert C.cal_max_gap({**OPT, "e_del": 2, "e_ins": 3}, 20) == 8    # (14/2 + 1, 14/3 + 1) -> 8
    assert C.cal_max_gap({**OPT, "e_del": 0}, 20) == 200              # x / 0 -> +inf -> i32::MAX -> 2w
    assert C.cal_max_gap({**OPT, "o_del": 30, "o_ins": 30, "e_del": 4, "e_ins": 4}, 25) == 1  # (-5/4 + 1) -> 0


def test_packed_reference_both_strands(built):
    from ferrousalign_b200.collect import pack_reference
    codes = np.array([0, 1, 2, 3, 3, 2, 1, 0, 2, 2, 1], np.uint8)
    pac, l_pac = pack_reference(codes)
    assert l_pac == 11 and len(pac) == 3
    assert pac[0] == 0b00011011                    # A C G T, first base in the high bits
    assert C.reference_segment(pac, l_pac, 2, 5) == [2, 3, 3, 2, 1]
    # reverse strand: position p >= l_pac is the complement of forward 2 l_pac - 1 - p
    rc = [3 - int(b) for b in codes[::-1]]
    assert C.reference_segment(pac, l_pac, l_pac, l_pac) == rc
    assert C.reference_segment(pac, l_pac, l_pac + 3, 4) == rc[3:7]
    assert C.reference_segment(pac, l_pac, 9, 4) == []     # across l_pac: empty


def test_jobs_of_a_hand_chain(built):
    from ferrousalign_b200.collect import pack_reference
    rng = np.random.default_rng(0)
    ref = rng.integers(0, 4, 2000).astype(np.uint8)
    pac, l_pac = pack_reference(ref)
    read = list(ref[500:560])                   # 60 bp from forward position 500
    chains = [{"read": 0, "seed_first": 0, "n_seeds": 2, "kept": 1},
              {"read": 0, "seed_first": 2, "n_seeds": 1, "kept": 0}]
    seeds = [{"ref_pos": 510, "query_pos": 10, "len": 20}, {"ref_pos": 540, "query_pos": 40, "len": 20},
             {"ref_pos": 700, "query_pos": 0, "len": 30}]
    out = C.collect(OPT, pac, l_pac, [read], chains, seeds)
    # window: seed 0 -> [510 - (10 + 5), 530 + (30 + 25)) = [495, 585); seed 1 -> [540 - (40 + 35), 560 + 1);
    # together [465, 585)
    assert out["chain_win"] == [(465, 585), (0, 0)]
    assert out["chain_first"] == [0, 2, 2]
    # seeds last to first: seed 1 first (left job 0; ends at the read end: no right job)
    t0, t1 = out["seed_ext"]
    assert (t0["ref_pos"], t0["left_job"], t0["right_job"]) == (540, 0, -1)
    assert (t1["ref_pos"], t1["left_job"], t1["right_job"]) == (510, 1, 0)
    q, t, h0, w, d = out["left"][0]
    assert q == read[:40][::-1] and t == list(ref[465:540][::-1]) and (h0, w, d) == (20, 100, 0)
    q, t, h0, w, d = out["right"][0]
    assert q == read[30:] and t == list(ref[530:585]) and (h0, w, d) == (0, 100, 1)


def test_window_cut_to_the_first_seeds_strand(built):
    from ferrousalign_b200.collect import pack_reference
    ref = np.arange(200, dtype=np.uint8) % 4
    pac, l_pac = pack_reference(ref)
    read = [0] * 50
    # a forward seed near the end of the forward strand: the window would cross l_pac
    seeds = [{"ref_pos": 190, "query_pos": 0, "len": 5}]
    out = C.collect(OPT, pac, l_pac, [read], [{"read": 0, "seed_first": 0, "n_seeds": 1, "kept": 1}], seeds)
    assert out["chain_win"] == [(189, 200)]      # [190 - 1, 190 + 5 + 85) cut at l_pac
    # the same seed on the reverse strand keeps the window above l_pac
    seeds = [{"ref_pos": 201, "query_pos": 20, "len": 5}]
    out = C.collect(OPT, pac, l_pac, [read], [{"read": 0, "seed_first": 0, "n_seeds": 1, "kept": 1}], seeds)
    assert out["chain_win"] == [(200, 251)]      # [201 - 35, 201 + 5 + 45) cut at l_pac
