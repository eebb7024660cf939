"""The CIGAR kernel (csrc/cigar_kernel.cu) against the CPU restatement of scalar_banded_swa
(oracle/cigar_oracle.py): scores and ends, every CIGAR operation and both aligned base
strings, on extension-shaped jobs at several bands, uneven jobs with N bases and repeats,
codes above 4, empty sequences and a zero band.  Bit-exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def oracle_params(p):
    return {"mat": [int(x) for x in p["mat"][0]], "o_del": int(p["o_del"][0]), "e_del": int(p["e_del"][0]),
            "o_ins": int(p["o_ins"][0]), "e_ins": int(p["e_ins"][0]), "zdrop": int(p["zdrop"][0]),
            "pen_clip3": int(p["pen_clip3"][0])}


def check(p, jobs, qseq, tseq):
    from ferrousalign_b200 import cigar as G
    from oracle import cigar_oracle as C
    got = G.scalar_banded_swa_batch(p, jobs, qseq, tseq)
    op = oracle_params(p)
    for k, j in enumerate(jobs):
        q = qseq[int(j["q_off"]):int(j["q_off"]) + int(j["qlen"])]
        t = tseq[int(j["t_off"]):int(j["t_off"]) + int(j["tlen"])]
        out, cig, ra, qa = C.banded_swa(op, list(q), list(t), int(j["w"]), int(j["h0"]))
        r = got.results[k]
        assert {f: int(r[f]) for f in out} == out, (k, r, out)
        assert got.cigar_of(k) == cig, (k, got.cigar_of(k), cig)
        assert list(got.ref_aligned_of(k)) == ra and list(got.query_aligned_of(k)) == qa, k
    return got


def jobs_from(batch, rng, bands=(0, 5, 20, 100), h0s=(0,)):
    from ferrousalign_b200 import cigar as G
    j = np.zeros(len(batch.jobs), G.CIGAR_JOB_DT)
    j["q_off"], j["t_off"] = batch.jobs["q_off"], batch.jobs["t_off"]
    j["qlen"], j["tlen"] = batch.jobs["qlen"], batch.jobs["tlen"]
    j["w"] = rng.choice(bands, len(j))
    j["h0"] = rng.choice(h0s, len(j))
    return j


def test_extension_shaped_jobs(built):
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import synth
    rng = np.random.default_rng(1)
    b = synth.workload_ext_1m(600)
    p = fa.BandedPairWiseSW().to_struct()
    got = check(p, jobs_from(b, rng, h0s=(0, 0, 19, 40)), b.qseq, b.tseq)
    assert (got.results["n_cigar"] > 0).all()


def test_uneven_jobs_other_scoring(built):
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import synth
    rng = np.random.default_rng(2)
    b = synth.workload_ext_uneven(500, ref_len=2_000_000)
    sw = fa.BandedPairWiseSW(o_del=5, e_del=2, o_ins=3, e_ins=1, zdrop=40, mat=fa.bwa_fill_scmat(2, 3, 0))
    p = sw.to_struct()
    p["pen_clip3"] = 9
    check(p, jobs_from(b, rng, bands=(3, 17, 60)), b.qseq, b.tseq)


def test_wide_scores_and_long_reads_take_the_int32_row_state(built):
    """A batch whose scores could pass 13 bits runs the 16-bit row state without query codes,
    one whose scores could pass 16 bits (h0 near 32767), or with a query longer than the
    shared row state holds, the int32 global-memory form: same results."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import synth
    rng = np.random.default_rng(4)
    b = synth.workload_ext_1m(300)
    p = fa.BandedPairWiseSW().to_struct()
    j = jobs_from(b, rng, bands=(5, 20))
    j["h0"][::7] = 10000           # past 13 bits: 16-bit row state without the query codes
    check(p, j, b.qseq, b.tseq)
    j["h0"][::7] = 32700           # past 16 bits: the int32 global row state
    check(p, j, b.qseq, b.tseq)
    ub = synth.workload_ext_uneven(200, ref_len=2_000_000)
    long_q = rng.integers(0, 4, 450).astype(np.uint8)
    qseq = np.concatenate([ub.qseq, long_q])
    tseq = np.concatenate([ub.tseq, long_q, rng.integers(0, 4, 40).astype(np.uint8)])
    j2 = jobs_from(ub, rng, bands=(3, 17))
    extra = np.zeros(1, j2.dtype)
    extra[0] = (len(ub.qseq), len(ub.tseq), 450, 490, 30, 0)
    check(p, np.concatenate([j2, extra]), qseq, tseq)


def test_wide_band_over_long_targets(built):
    """w = 100 over 1000-base targets (the row state's full band, rows far past the query's
    length): same results as the oracle."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import cigar as G
    rng = np.random.default_rng(5)
    qs, ts, jobs = [], [], np.zeros(3, G.CIGAR_JOB_DT)
    qo = to = 0
    for k in range(3):
        t = rng.integers(0, 4, 1000).astype(np.uint8)
        q = t[300 + 50 * k:500 + 50 * k].copy()
        q[rng.integers(0, 200, 6)] = rng.integers(0, 4, 6)
        jobs[k] = (qo, to, len(q), len(t), 100, 0)
        qs.append(q); ts.append(t); qo += len(q); to += len(t)
    check(fa.BandedPairWiseSW().to_struct(), jobs, np.concatenate(qs), np.concatenate(ts))


def test_edges_codes_and_empty(built):
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import cigar as G
    rng = np.random.default_rng(3)
    n = 200
    ql = rng.integers(0, 60, n)
    tl = rng.integers(0, 70, n)
    ql[:5] = 0
    tl[5:10] = 0
    qseq = rng.integers(0, 8, int(ql.sum()) + 1).astype(np.uint8)    # codes 5-7 count as N
    tseq = rng.integers(0, 8, int(tl.sum()) + 1).astype(np.uint8)
    jobs = np.zeros(n, G.CIGAR_JOB_DT)
    jobs["q_off"] = np.concatenate([[0], np.cumsum(ql)[:-1]])
    jobs["t_off"] = np.concatenate([[0], np.cumsum(tl)[:-1]])
    jobs["qlen"], jobs["tlen"] = ql, tl
    jobs["w"] = rng.integers(0, 40, n)
    jobs["h0"] = rng.integers(0, 30, n)
    # similar pairs too: the target a mutated copy of the query
    for k in range(100, n):
        q = qseq[int(jobs["q_off"][k]):int(jobs["q_off"][k]) + int(ql[k])]
        m = min(int(ql[k]), int(tl[k]))
        tseq[int(jobs["t_off"][k]):int(jobs["t_off"][k]) + m] = q[:m]
    got = check(fa.BandedPairWiseSW().to_struct(), jobs, qseq, tseq)
    assert (got.results["n_cigar"][:10] == 0).all()


def test_packed_and_slotted_layouts_agree(built):
    """fa_cigar_batch_packed gives the slotted call's words back to back (offsets = running
    sums of n_cigar); a buffer one word short returns FA_ERR_CAPACITY with the results and
    offsets filled."""
    import ctypes
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N, cigar as G, synth
    rng = np.random.default_rng(5)
    b = synth.workload_ext_uneven(3000, ref_len=2_000_000)
    jobs = jobs_from(b, rng, bands=(0, 3, 17, 60))
    p = fa.BandedPairWiseSW().to_struct()
    pk = G.scalar_banded_swa_batch(p, jobs, b.qseq, b.tseq, packed=True)
    sl = G.scalar_banded_swa_batch(p, jobs, b.qseq, b.tseq, packed=False)
    assert np.array_equal(pk.results, sl.results)
    n_cig = sl.results["n_cigar"].astype(np.uint64)
    assert np.array_equal(pk.cigar_off, np.concatenate([[0], np.cumsum(n_cig)[:-1]]).astype(np.uint64))
    assert len(pk.cigar) == int(n_cig.sum())
    for k in range(len(jobs)):
        assert pk.cigar_of(k) == sl.cigar_of(k), k
        assert np.array_equal(pk.ref_aligned_of(k), sl.ref_aligned_of(k))
        assert np.array_equal(pk.query_aligned_of(k), sl.query_aligned_of(k))
    lib = N.load()
    ctx = N.default_context()
    n = len(jobs)
    res = np.zeros(n, G.CIGAR_RESULT_DT)
    first = np.zeros(n, np.uint64)
    cap = int(n_cig.sum()) - 1
    cig = np.zeros(cap, np.uint32)
    ra = np.zeros(int(jobs["tlen"].sum()) + 1, np.uint8)
    qa = np.zeros(int(jobs["qlen"].sum()) + 1, np.uint8)
    rc = lib.fa_cigar_batch_packed(ctx.handle, N.ptr(p), N.ptr(jobs), n, N.ptr(b.qseq), len(b.qseq), N.ptr(b.tseq),
                                   len(b.tseq), N.ptr(res), N.ptr(cig), ctypes.c_uint64(cap), N.ptr(first),
                                   N.ptr(ra), N.ptr(qa))
    assert rc == N.FA_ERR_CAPACITY
    assert np.array_equal(res, sl.results) and np.array_equal(first, pk.cigar_off)
