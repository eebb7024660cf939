"""Soundness of the exit-bound certificate, checked on the CPU oracle.

A narrow run (band w) that certifies must reproduce the run at the configured band W
on every output field.  The certificate is a proof obligation of the learned-band
path's exactness; these cases exercise it on seeded workloads with several read-length
regimes, indel rates, scorings, z-drop settings and both extension directions.
"""
import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from ferrousalign_b200 import synth
from oracle import ksw_oracle as O


def scoring(a=1, b=4, o_del=6, e_del=1, o_ins=6, e_ins=1, zdrop=100, end_bonus=5):
    p = np.zeros(1, N.PARAMS_DT)
    p["mat"][0] = fa.bwa_fill_scmat(a, b).astype(np.int8).ravel()
    p["m"] = 5
    p["o_del"], p["e_del"], p["o_ins"], p["e_ins"] = o_del, e_del, o_ins, e_ins
    p["zdrop"], p["end_bonus"] = zdrop, end_bonus
    return p


def batch_151(n, seed, **kw):
    ref = synth.reference(200_000, seed=seed)
    return synth.ext_jobs(ref, n, seed=seed + 1, **kw)


CASES = {
    "151bp_mixture": (lambda: batch_151(6000, 41, indel_rates=(0.0, 0.001, 0.01, 0.03)), scoring()),
    "indel_heavy": (lambda: batch_151(4000, 43, indel_rates=(0.05,), indel_mean=3.0), scoring()),
    "uneven_left_right": (lambda: synth.ext_jobs(synth.reference(300_000, seed=45, repeat_frac=0.05), 4000,
                                                 seed=46, read_len=(50, 300), seed_at_start=False), scoring()),
    "short_seeds": (lambda: batch_151(4000, 47, seed_len=(5, 12), sub_rate=0.03), scoring()),
    "match2_gaps": (lambda: batch_151(4000, 49, match_score=2, indel_rates=(0.01,)),
                    scoring(a=2, b=5, o_del=5, e_del=2, o_ins=4, e_ins=3, zdrop=60, end_bonus=0)),
    "no_zdrop": (lambda: batch_151(4000, 51, indel_rates=(0.01,), sub_rate=0.04), scoring(zdrop=0)),
    "cheap_gaps": (lambda: batch_151(4000, 53, indel_rates=(0.03,)), scoring(o_del=2, e_del=1, o_ins=1, e_ins=1)),
}


def certified(p, jobs, out, tr):
    ok = tr["bound_ok"].astype(bool)
    clean = np.array([O.wide_clean(p, int(j["qlen"]), int(j["w"]), int(r)) for j, r in zip(jobs, tr["init_reach"])])
    return ok & clean


@pytest.mark.parametrize("name", sorted(CASES))
def test_certified_runs_equal_configured_band(name):
    make, p = CASES[name]
    b = make()
    ref, _ = O.ext_batch(p, b.jobs, b.qseq, b.tseq)
    total = 0
    for w in (1, 2, 4, 8, 16, 32, 64):
        j = b.jobs.copy()
        j["w"] = np.minimum(j["w"], w)
        out, tr = O.ext_batch(p, j, b.qseq, b.tseq)
        c = certified(p, b.jobs, out, tr)
        bad = np.nonzero(c & (out != ref))[0]
        assert len(bad) == 0, f"{name} w={w}: certified but different at jobs {bad[:5]}"
        total += int(c.sum())
    assert total > 0, "the certificate never fired"


@pytest.mark.parametrize("name", ["151bp_mixture", "uneven_left_right", "match2_gaps"])
def test_bound_policy_equals_plain_policy(name):
    make, p = CASES[name]
    b = make()
    plain, _, _, pc = O.ext_batch_policy(p, fa.make_policy(N.FA_POLICY_BWA, 2), b.jobs, b.qseq, b.tseq)
    rng = np.random.default_rng(5)
    wf = rng.choice([1, 2, 4, 8, 16, 32], len(b.jobs)).astype(np.int32)
    for judge in (N.FA_JUDGE_BOUND, N.FA_JUDGE_BOUND | N.FA_JUDGE_ONCE,
                  N.FA_JUDGE_BOUND | N.FA_JUDGE_ONCE | N.FA_JUDGE_HINT):
        pol = fa.make_policy(N.FA_POLICY_LEARNED, 2, judge, 1)
        out, wfin, tries, cells = O.ext_batch_policy(p, pol, b.jobs, b.qseq, b.tseq, wf)
        assert np.array_equal(out, plain)
        assert (wfin < b.jobs["w"]).mean() > 0.3          # most jobs stop at a narrow band
        assert cells.sum() < pc.sum()
        if judge & N.FA_JUDGE_HINT:                       # some rejected runs retried narrow
            assert ((tries == 2) & (wfin < b.jobs["w"])).any()


def test_certificate_examples():
    """A clean read certifies at a narrow band; a read with many mismatches does not."""
    p = scoring()
    rng = np.random.default_rng(3)
    t = rng.integers(0, 4, 220).astype(np.uint8)
    q = t[:120].copy()
    out_n, tr = O.ksw_extend2(q, t, p["mat"][0], 6, 1, 6, 1, 8, 5, 100, 40)
    out_w, _ = O.ksw_extend2(q, t, p["mat"][0], 6, 1, 6, 1, 100, 5, 100, 40)
    assert tr["bound_ok"] == 1 and out_n == out_w
    q2 = q.copy()
    q2[10:120:12] = (q2[10:120:12] + 1) % 4          # ten mismatches
    _, tr2 = O.ksw_extend2(q2, t, p["mat"][0], 6, 1, 6, 1, 8, 5, 100, 40)
    assert tr2["bound_ok"] == 0
