"""Extension kernel parity: the CUDA path through the C ABI against the CPU oracle,
bit-exact on all six KswExtendResult fields."""
import json
from pathlib import Path

import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from ferrousalign_b200 import synth
from oracle import ksw_oracle as O

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def params_of(c):
    p = np.zeros(1, N.PARAMS_DT)
    p["mat"][0] = np.array(c["mat"], np.int8)
    p["m"] = 5
    for k in ("o_del", "e_del", "o_ins", "e_ins", "zdrop", "end_bonus"):
        p[k] = c[k]
    return p


def one_job_arrays(q, t, h0, w):
    jobs = np.zeros(1, N.JOB_DT)
    jobs[0] = (0, 0, len(q), len(t), h0, w, 1, 0)
    qa = np.array(q if len(q) else [0], np.uint8)
    ta = np.array(t if len(t) else [0], np.uint8)
    return jobs, qa, ta


def diff_report(a, b):
    bad = np.nonzero(a != b)[0]
    return f"{len(bad)} mismatches, first {bad[:5]}: gpu={a[bad[:3]]} oracle={b[bad[:3]]}"


@pytest.mark.parametrize("case", json.loads((GOLD / "ext_cases.json").read_text()), ids=lambda c: c["name"])
def test_golden_case(ctx, case):
    jobs, q, t = one_job_arrays(case["query"], case["target"], case["h0"], case["w"])
    out, _, _ = fa.extend_batch(params_of(case), jobs, q, t, ctx=ctx)
    assert list(out[0]) == case["expect"]


def run_both(ctx, p, b, threads=0):
    out, stats, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, ctx=ctx)
    ref, tr = O.ext_batch(p, b.jobs, b.qseq, b.tseq, threads=threads)
    return out, stats, ref, tr


def test_plain_10k_bit_exact(ctx):
    b = synth.workload_ext_plain(10_000)
    p = fa.BandedPairWiseSW().to_struct()
    out, stats, ref, tr = run_both(ctx, p, b)
    assert np.array_equal(out, ref), diff_report(out, ref)
    assert stats["cells"] == tr["cells"].sum()      # same visited-cell count as the oracle


def test_indel_mixture_200k_bit_exact(ctx):
    b = synth.workload_ext_1m(200_000)
    p = fa.BandedPairWiseSW().to_struct()
    out, stats, ref, tr = run_both(ctx, p, b)
    assert np.array_equal(out, ref), diff_report(out, ref)
    assert stats["cells"] == tr["cells"].sum()


def test_uneven_left_right_bit_exact(ctx):
    ref_seq = synth.reference(20_000_000, seed=3, n_rate=0.001, repeat_frac=0.05)
    b = synth.ext_jobs(ref_seq, 60_000, seed=103, read_len=(50, 300), seed_at_start=False)
    p = fa.BandedPairWiseSW().to_struct()
    out, _, ref, _ = run_both(ctx, p, b)
    assert np.array_equal(out, ref), diff_report(out, ref)


@pytest.mark.parametrize("a,b_,n,gaps,w,zdrop,eb", [
    (1, 4, -1, (6, 1, 6, 1), 100, 100, 5),
    (2, 3, 0, (5, 2, 3, 1), 30, 40, 0),
    (1, 1, -2, (0, 1, 0, 1), 10, 0, 5),
    (3, 5, -1, (6, 1, 4, 3), 5, 20, 10),
    (1, 4, -1, (4, 0, 4, 1), 50, 100, 5),
])
def test_parameter_sweep_bit_exact(ctx, a, b_, n, gaps, w, zdrop, eb):
    ref_seq = synth.reference(500_000, seed=11, n_rate=0.01)
    b = synth.ext_jobs(ref_seq, 20_000, seed=17, read_len=(30, 200), seed_len=(5, 40), w=w,
                       indel_rates=(0.0, 0.01, 0.05), sub_rate=0.03)
    sw = fa.BandedPairWiseSW(o_del=gaps[0], e_del=gaps[1], o_ins=gaps[2], e_ins=gaps[3], zdrop=zdrop,
                             end_bonus=eb, mat=fa.bwa_fill_scmat(a, b_, n))
    p = sw.to_struct()
    out, _, ref, _ = run_both(ctx, p, b)
    assert np.array_equal(out, ref), diff_report(out, ref)


@pytest.mark.parametrize("kernel,threads", [(N.FA_KERNEL_INT32, 64), (N.FA_KERNEL_INT32, 128),
                                            (N.FA_KERNEL_INT32, 256), (N.FA_KERNEL_INT16X2, 128),
                                            (N.FA_KERNEL_ROWS2, 64), (N.FA_KERNEL_ROWS2, 128)])
def test_kernel_variants_bit_exact(ctx, kernel, threads):
    """Every autotuning candidate (int32 one job per thread at 64/128/256 threads per
    block, int16x2 two jobs per thread, int16x2 two target rows per thread at 64/128)
    gives the oracle's results, including reads past 254 bases and a = 3 scoring, where
    the two-row kernel hands jobs on to the int32 kernel."""
    b = synth.workload_ext_1m(100_000, seed=31)
    p = fa.BandedPairWiseSW().to_struct()
    ctx.set_kernel(kernel)
    ctx.set_threads(threads)
    try:
        out, stats, ref, tr = run_both(ctx, p, b)
        ref_seq = synth.reference(5_000_000, seed=6, n_rate=0.01, repeat_frac=0.05)
        u = synth.ext_jobs(ref_seq, 30_000, seed=66, read_len=(20, 300), seed_at_start=False, seed_len=(10, 40))
        out2, _, ref2, _ = run_both(ctx, p, u)
        sw = fa.BandedPairWiseSW(o_del=5, e_del=2, o_ins=3, e_ins=1, mat=fa.bwa_fill_scmat(3, 2, 0), zdrop=30)
        out3, _, ref3, _ = run_both(ctx, sw.to_struct(), u)
        choice = ctx.kernel_choice()
    finally:
        ctx.set_kernel(N.FA_KERNEL_AUTO)
        ctx.set_threads(128)
    assert choice["kernel"] == {N.FA_KERNEL_INT32: "int32", N.FA_KERNEL_INT16X2: "int16x2",
                                N.FA_KERNEL_ROWS2: "rows2"}[kernel]
    assert np.array_equal(out, ref), diff_report(out, ref)
    assert stats["cells"] == tr["cells"].sum()
    assert np.array_equal(out2, ref2), diff_report(out2, ref2)
    assert np.array_equal(out3, ref3), diff_report(out3, ref3)


def test_policies_match_oracle(ctx):
    b = synth.workload_ext_1m(30_000, seed=21)
    p = fa.BandedPairWiseSW().to_struct()
    pol = fa.make_policy(N.FA_POLICY_BWA, 2)
    out, st, wfin = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=pol, ctx=ctx)
    ref, rwfin, rtries, _ = O.ext_batch_policy(p, pol, b.jobs, b.qseq, b.tseq)
    assert np.array_equal(out, ref), diff_report(out, ref)
    assert np.array_equal(wfin, rwfin)
    assert st["retries"] == (rtries - 1).sum()
    rng = np.random.default_rng(5)
    wf = rng.choice([5, 10, 20, 40], size=len(b.jobs)).astype(np.int32)
    for judge in (N.FA_JUDGE_CERT, N.FA_JUDGE_CERT | N.FA_JUDGE_MAXOFF, N.FA_JUDGE_BOUND):
        pol = fa.make_policy(N.FA_POLICY_LEARNED, 2, judge, 1)
        out, st, wfin = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=pol, w_first=wf, ctx=ctx)
        ref, rwfin, rtries, _ = O.ext_batch_policy(p, pol, b.jobs, b.qseq, b.tseq, wf)
        assert np.array_equal(out, ref), diff_report(out, ref)
        assert np.array_equal(wfin, rwfin)     # same acceptance decisions, so the same certificates


@pytest.mark.parametrize("workload", ["mixture", "uneven"])
def test_bound_judge_is_exact_and_matches_oracle(ctx, workload):
    """Narrow bands accepted by the exit-bound certificate reproduce the plain
    policy bit for bit; the GPU takes the same decisions as the oracle."""
    if workload == "mixture":
        b = synth.workload_ext_1m(100_000, seed=23)
    else:
        b = synth.workload_ext_uneven(50_000, seed=24, ref_len=5_000_000)
    p = fa.BandedPairWiseSW().to_struct()
    plain, pst, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=fa.make_policy(N.FA_POLICY_BWA, 2), ctx=ctx)
    rng = np.random.default_rng(7)
    wf = rng.choice([2, 4, 8, 16, 32], size=len(b.jobs)).astype(np.int32)
    for judge in (N.FA_JUDGE_BOUND, N.FA_JUDGE_BOUND | N.FA_JUDGE_ONCE | N.FA_JUDGE_HINT):
        pol = fa.make_policy(N.FA_POLICY_LEARNED, 2, judge, 1)
        out, st, wfin = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=pol, w_first=wf, ctx=ctx)
        assert np.array_equal(out, plain), diff_report(out, plain)
        ref, rwfin, rtries, rcells = O.ext_batch_policy(p, pol, b.jobs, b.qseq, b.tseq, wf)
        assert np.array_equal(wfin, rwfin)          # same certificates and the same hints
        assert st["cells_executed"] == rcells.sum()
        assert st["cells_executed"] < pst["cells_executed"]


def test_reference_style_interface(ctx):
    batch = fa.ExtensionJobBatch()
    sw = fa.BandedPairWiseSW()
    rng = np.random.default_rng(3)
    for k in range(50):
        q = rng.integers(0, 4, 80).astype(np.uint8)
        t = np.concatenate([q, rng.integers(0, 4, 60).astype(np.uint8)])
        batch.add_job(k, 0, 0, fa.ExtensionDirection.Right, q, t, 20, 100)
    res = fa.execute_batch_simd_scoring(sw, batch)
    assert len(res) == 50
    for k, r in enumerate(res):
        o, _ = O.ksw_extend2(batch.get_query_seq(k), batch.get_ref_seq(k), sw.mat, 6, 1, 6, 1, 100, 5, 100, 20)
        assert (r.score, r.query_end, r.ref_end, r.gref_end, r.gscore, r.max_off) == tuple(o)
        assert r.read_idx == k
    assert fa.execute_batch_simd_scoring(sw, fa.ExtensionJobBatch()) == []


def test_errors_are_reported(ctx):
    p = fa.BandedPairWiseSW().to_struct()
    jobs, q, t = one_job_arrays([0, 1, 2], [0, 1, 2], 0, 100)        # h0 = 0 panics in the reference
    with pytest.raises(N.NativeError) as e:
        fa.extend_batch(p, jobs, q, t, ctx=ctx)
    assert e.value.code == N.FA_ERR_ARG
    jobs, q, t = one_job_arrays([0, 7, 2], [0, 1, 2], 5, 100)        # code outside the alphabet
    with pytest.raises(N.NativeError) as e:
        fa.extend_batch(p, jobs, q, t, ctx=ctx)
    assert e.value.code == N.FA_ERR_ARG
    jobs, q, t = one_job_arrays([0, 1, 2], [0, 1, 2], 5, 100)
    jobs["t_off"] = 10                                               # range outside the buffer
    with pytest.raises(N.NativeError) as e:
        fa.extend_batch(p, jobs, q, t, ctx=ctx)
    assert e.value.code == N.FA_ERR_ARG
    jobs, q, t = one_job_arrays([0] * 10, [0] * 10, 9000, 100)       # beyond the packed-column bound
    with pytest.raises(N.NativeError) as e:
        fa.extend_batch(p, jobs, q, t, ctx=ctx)
    assert e.value.code == N.FA_ERR_CAPACITY
    # the context stays usable after errors
    jobs, q, t = one_job_arrays([0, 1, 2, 3], [0, 1, 2, 3], 10, 50)
    out, _, _ = fa.extend_batch(p, jobs, q, t, ctx=ctx)
    assert out[0]["qle"] == 4 and out[0]["tle"] == 4


def test_large_batch_errors_and_pinned_pipeline(ctx):
    """Batches large enough for the sliced-upload path: the first bad job is reported with
    the same code and message as on the serial path, nothing runs, the context stays
    usable, and pinned host buffers give the serial path's results."""
    import torch
    p = fa.BandedPairWiseSW().to_struct()
    b = synth.workload_ext_1m(60_000, seed=31)
    for field, value, code in (("q_off", 10 ** 12, N.FA_ERR_ARG), ("h0", 0, N.FA_ERR_ARG),
                               ("qlen", 5000, N.FA_ERR_CAPACITY)):
        jobs = b.jobs.copy()
        jobs[40_001][field] = value
        jobs[51_234][field] = value
        with pytest.raises(N.NativeError) as e:
            fa.extend_batch(p, jobs, b.qseq, b.tseq, ctx=ctx)
        assert e.value.code == code and "job 40001" in str(e.value)
    ref, tr = O.ext_batch(p, b.jobs, b.qseq, b.tseq)
    pin_q = torch.from_numpy(b.qseq).pin_memory().numpy()
    pin_t = torch.from_numpy(b.tseq).pin_memory().numpy()
    pin_j = torch.from_numpy(b.jobs.view(np.uint8)).pin_memory().numpy().view(N.JOB_DT)
    for _ in range(2):
        out, st, _ = fa.extend_batch(p, pin_j, pin_q, pin_t, ctx=ctx)
        assert np.array_equal(out, ref), diff_report(out, ref)
        assert st["cells"] == tr["cells"].sum()


def test_autotuner_picks_a_measured_candidate():
    """FA_KERNEL_AUTO times every candidate once per shape and runs the fastest; the
    results equal the oracle's whichever wins."""
    b = synth.workload_ext_1m(150_000, seed=33)
    p = fa.BandedPairWiseSW().to_struct()
    c = N.Context(0)
    try:
        out, _, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, ctx=c)
        ch = c.kernel_choice()
        cands = ch["candidates"]
        assert len(cands) >= 3
        best = min(cands, key=lambda x: x["sample_ms"])
        assert (best["kernel"], best["threads_per_block"]) == (ch["kernel"], ch["threads_per_block"])
        out2, _, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, ctx=c)   # cached choice, no new table
        assert c.kernel_choice()["kernel"] == ch["kernel"]
    finally:
        c.close()
    ref, _ = O.ext_batch(p, b.jobs, b.qseq, b.tseq)
    assert np.array_equal(out, ref) and np.array_equal(out2, ref)


@pytest.mark.gpu
def test_rows2_under_retry_policy_and_graph():
    """The two-row kernel inside the bwa-mem2 retry rounds (device job counts, per-job
    bands) and as a recorded CUDA graph: the oracle's results and bands."""
    b = synth.workload_ext_1m(40_000, seed=35)
    p = fa.BandedPairWiseSW(zdrop=40).to_struct()
    pol = fa.make_policy(N.FA_POLICY_BWA, 2)
    ref, rwfin, _, _ = O.ext_batch_policy(p, pol, b.jobs, b.qseq, b.tseq)
    c = N.Context(0)
    try:
        c.set_kernel(N.FA_KERNEL_ROWS2)
        out, _, wfin = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=pol, ctx=c)
        c.set_graph(True)
        outg, _, wfing = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=pol, ctx=c)
        outg2, _, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=pol, ctx=c)
        assert c.kernel_choice()["kernel"] == "rows2"
    finally:
        c.close()
    for o, wf in ((out, wfin), (outg, wfing), (outg2, wfing)):
        assert np.array_equal(o, ref), diff_report(o, ref)
        assert np.array_equal(wf, rwfin)
