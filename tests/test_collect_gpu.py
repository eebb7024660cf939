"""The job-collection kernels (csrc/collect_kernel.cu) against the CPU restatement of
collect_extension_jobs_batch_soa (oracle/collect_oracle.py): every job's query and target
bases, h0, band and direction, the seed table, the chain windows; then the whole
chain -> jobs -> extension -> region path against the oracle's.  Bit-exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def oracle_collect(opts, pac, l_pac, reads, read_off, chains, seeds):
    from oracle import collect_oracle as C
    o = {k: int(opts[k][0]) for k in ("a", "o_del", "e_del", "o_ins", "e_ins", "w")}
    rl = [list(reads[int(read_off[r]):int(read_off[r + 1])]) for r in range(len(read_off) - 1)]
    ch = [{k: int(c[k]) for k in ("read", "seed_first", "n_seeds", "kept")} for c in chains]
    sd = [{"ref_pos": int(s["ref_pos"]), "query_pos": int(s["query_pos"]), "len": int(s["len"])} for s in seeds]
    return C.collect(o, pac, l_pac, rl, ch, sd)


def check_same(got, want):
    for side, jobs in (("left", got.left_jobs), ("right", got.right_jobs)):
        ref = want[side]
        assert len(jobs) == len(ref), side
        for j, (q, t, h0, w, d) in zip(jobs, ref):
            assert (int(j["h0"]), int(j["w"]), int(j["dir"])) == (h0, w, d)
            assert list(got.qbuf[int(j["q_off"]):int(j["q_off"]) + int(j["qlen"])]) == q
            assert list(got.tbuf[int(j["t_off"]):int(j["t_off"]) + int(j["tlen"])]) == t
    ext = want["seed_ext"]
    assert len(got.seed_ext) == len(ext)
    for e, r in zip(got.seed_ext, ext):
        assert tuple(int(e[k]) for k in ("ref_pos", "query_pos", "len", "left_job", "right_job")) == \
            tuple(r[k] for k in ("ref_pos", "query_pos", "len", "left_job", "right_job"))
    assert list(got.chain_first) == want["chain_first"]
    assert [tuple(int(x) for x in w) for w in got.chain_win] == want["chain_win"]


def test_chains_of_both_strands_match_oracle(built):
    from ferrousalign_b200 import collect as K, synth
    ref, reads, off, chains, seeds = synth.workload_chains(3000, ref_len=2_000_000)
    pac, l_pac = K.pack_reference(ref)
    for opts in (K.collect_opts(), K.collect_opts(a=2, o_del=5, e_del=2, o_ins=4, e_ins=0, w=30)):
        got = K.collect_extension_jobs(pac, l_pac, reads, off, chains, seeds, opts=opts)
        want = oracle_collect(opts, pac, l_pac, reads, off, chains, seeds)
        assert len(want["left"]) > 1000 and len(want["right"]) > 1000
        check_same(got, want)


def test_chain_to_region_path(built):
    """Collected jobs through the extension kernels (right jobs with the seed's score as h0,
    the bwa-mem2 form: h0 = 0 is outside ksw_extend2's contract) and the region merge, the
    same jobs through the oracle's extension and merge."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import collect as K, synth
    from oracle import ksw_oracle as O, region_oracle as R
    ref, reads, off, chains, seeds = synth.workload_chains(4000, ref_len=2_000_000)
    pac, l_pac = K.pack_reference(ref)
    got = K.collect_extension_jobs(pac, l_pac, reads, off, chains, seeds)
    p = fa.BandedPairWiseSW().to_struct()
    right = got.right_jobs.copy()
    owner = np.full(len(right), -1)
    for e in got.seed_ext:
        if e["right_job"] >= 0:
            owner[e["right_job"]] = e["len"]
    right["h0"] = owner
    assert (right["h0"] > 0).all()
    lres, _, _ = fa.extend_batch(p, got.left_jobs, got.qbuf, got.tbuf)
    rres, _, _ = fa.extend_batch(p, right, got.qbuf, got.tbuf)
    lref, _ = O.ext_batch(p, got.left_jobs, got.qbuf, got.tbuf)
    rref, _ = O.ext_batch(p, right, got.qbuf, got.tbuf)
    assert np.array_equal(lres, lref) and np.array_equal(rres, rref)
    qlen = np.diff(off.astype(np.int64))[chains["read"]].astype(np.int32)
    regions = fa.merge_scores_to_regions(got.chain_first, qlen, got.seed_ext, lres, rres)
    want = R.merge_regions({"a": 1, "pen_clip5": 5, "pen_clip3": 5, "w": 100}, got.chain_first, qlen,
                           got.seed_ext, lref, rref)
    assert np.array_equal(regions, want)
    assert (regions["seed"] >= 0).sum() > 0.9 * len(chains)


def test_argument_checks_and_capacity(built):
    from ferrousalign_b200 import _native as N, collect as K, synth
    ref, reads, off, chains, seeds = synth.workload_chains(200, ref_len=200_000)
    pac, l_pac = K.pack_reference(ref)
    lib = N.load()
    ctx = N.Context(0)
    opts = K.collect_opts()
    n = len(seeds)
    left, right = np.zeros(n, N.JOB_DT), np.zeros(n, N.JOB_DT)
    qbuf = np.zeros(2 * len(reads), np.uint8)
    tbuf = np.zeros(16, np.uint8)
    ext = np.zeros(n, N.SEED_EXT_DT)
    first = np.zeros(len(chains) + 1, np.uint32)
    win = np.zeros((len(chains), 2), np.uint64)
    counts = np.zeros(1, N.COLLECT_COUNTS_DT)

    def call(ch=chains, sd=seeds, cap=len(tbuf)):
        return lib.fa_collect_ext_jobs(ctx.handle, N.ptr(opts), N.ptr(pac), l_pac, N.ptr(reads), N.ptr(off),
                                       len(off) - 1, N.ptr(ch), len(ch), N.ptr(sd), len(sd), N.ptr(left),
                                       N.ptr(right), N.ptr(qbuf), N.ptr(tbuf), cap, N.ptr(ext), N.ptr(first),
                                       N.ptr(win), N.ptr(counts))
    assert call() == N.FA_ERR_CAPACITY and counts["tbuf_len"][0] > 16    # the bytes needed come back
    bad = seeds.copy()
    bad["query_pos"][0] = 200                                          # past its read
    assert call(sd=bad) == N.FA_ERR_ARG
    bad = seeds.copy()
    bad["ref_pos"][0] = 2 * l_pac                                      # past the reference
    assert call(sd=bad) == N.FA_ERR_ARG
    badc = chains.copy()
    badc["read"][0] = 10**6
    assert call(ch=badc) == N.FA_ERR_ARG

    def why(**kw):
        with pytest.raises(N.NativeError) as e:
            N.check(call(**kw))
        assert e.value.code == N.FA_ERR_ARG
        return str(e.value)
    # the first failing chain's first failing rule is reported, as a serial walk finds it
    kept = np.nonzero(chains["kept"] != 0)[0]
    k1, k2 = int(kept[3]), int(kept[7])
    badc = chains.copy()
    badc["seed_first"][k2] = len(seeds)                                # seeds past the array
    bad = seeds.copy()
    bad["ref_pos"][int(chains["seed_first"][k1])] = 2 * l_pac          # an earlier chain's seed
    assert "outside the reference" in why(ch=badc, sd=bad)
    assert "run past the seed array" in why(ch=badc)
    bad = seeds.copy()
    j = int(chains["seed_first"][k1])
    bad["ref_pos"][j] = 2 * l_pac
    bad["query_pos"][j] = 500
    assert "outside its read" in why(sd=bad)                           # the read rule is checked first
    ctx.close()


def test_packed_collection_equals_byte_collection(built):
    """fa_collect_ext_jobs_packed: the same jobs, seed table and chain windows as the byte
    form; its packed buffers unpack to the byte form's qbuf / tbuf (reads carrying N runs,
    at read edges too), and the jobs extend to the same results through the packed entry."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import collect as K, synth
    ref, reads, off, chains, seeds = synth.workload_chains(3000, ref_len=2_000_000)
    reads = reads.copy()
    rng = np.random.default_rng(11)
    for r in rng.choice(len(off) - 1, 200, replace=False):
        a, b = int(off[r]), int(off[r + 1])
        k = int(rng.integers(a, b))
        reads[k:min(b, k + int(rng.integers(1, 6)))] = 4
    reads[int(off[0])] = 4
    reads[int(off[-1]) - 1] = 4
    pac, l_pac = K.pack_reference(ref)
    byt = K.collect_extension_jobs(pac, l_pac, reads, off, chains, seeds)
    pk = K.collect_extension_jobs_packed(pac, l_pac, reads, off, chains, seeds)
    for f in ("left_jobs", "right_jobs", "seed_ext", "chain_first", "chain_win"):
        assert np.array_equal(getattr(pk, f), getattr(byt, f)), f
    assert np.array_equal(fa.unpack(pk.qbuf), byt.qbuf)
    assert np.array_equal(fa.unpack(pk.tbuf), byt.tbuf)
    assert len(pk.qbuf.runs) >= 200
    assert np.array_equal(pk.qbuf.runs, fa.packed.n_runs_of(byt.qbuf))
    p = fa.BandedPairWiseSW().to_struct()
    got, _, _ = fa.extend_batch_packed(p, pk.left_jobs, pk.qbuf, pk.tbuf)
    want, _, _ = fa.extend_batch(p, byt.left_jobs, byt.qbuf, byt.tbuf)
    assert np.array_equal(got, want)


def test_reused_pinned_buffers_give_fresh_results(built):
    """Collection and CIGAR regeneration into reused page-locked HostBuffers: two batches of
    different sizes, one after the other through the same buffers, equal the calls into
    fresh arrays (the outputs are written in full, so stale bytes of a larger earlier batch
    never show)."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import collect as K, synth
    bufs, pbufs, cbufs = fa.HostBuffers(), fa.HostBuffers(), fa.HostBuffers()
    p = fa.BandedPairWiseSW().to_struct()
    for n, seed in ((4000, 5), (2500, 6)):
        ref, reads, off, chains, seeds = synth.workload_chains(n, ref_len=2_000_000, seed=seed)
        pac, l_pac = K.pack_reference(ref)
        want = K.collect_extension_jobs(pac, l_pac, reads, off, chains, seeds)
        got = K.collect_extension_jobs(pac, l_pac, reads, off, chains, seeds, bufs=bufs)
        pk = K.collect_extension_jobs_packed(pac, l_pac, reads, off, chains, seeds, bufs=pbufs)
        for f in ("left_jobs", "right_jobs", "seed_ext", "chain_first", "chain_win", "qbuf", "tbuf"):
            assert np.array_equal(getattr(got, f), getattr(want, f)), f
        for f in ("left_jobs", "right_jobs", "seed_ext", "chain_first", "chain_win"):
            assert np.array_equal(getattr(pk, f), getattr(want, f)), f
        assert np.array_equal(fa.unpack(pk.tbuf), want.tbuf)
        cj, cq, ct = synth.workload_cigar(n, seed=seed)
        cw = fa.scalar_banded_swa_batch(p, cj, cq, ct)
        cg = fa.scalar_banded_swa_batch(p, cj, cq, ct, bufs=cbufs)
        assert np.array_equal(cg.results, cw.results)
        assert all(cg.cigar_of(i) == cw.cigar_of(i) for i in range(0, n, 97))


def test_resident_reference(built):
    """Context.set_reference keeps the packed reference on the device: collection calls given
    pac=None read it and equal the calls that upload it; a call whose l_pac differs from the
    resident copy's, or one after the copy is dropped, fails with FA_ERR_ARG."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N, collect as K, synth
    ref, reads, off, chains, seeds = synth.workload_chains(3000, ref_len=2_000_000, seed=9)
    pac, l_pac = K.pack_reference(ref)
    with fa.Context(0) as ctx:
        want = K.collect_extension_jobs(pac, l_pac, reads, off, chains, seeds, ctx=ctx)
        ctx.set_reference(pac, l_pac)
        got = K.collect_extension_jobs(None, l_pac, reads, off, chains, seeds, ctx=ctx)
        pk = K.collect_extension_jobs_packed(None, l_pac, reads, off, chains, seeds, ctx=ctx)
        for f in ("left_jobs", "right_jobs", "seed_ext", "chain_first", "chain_win", "qbuf", "tbuf"):
            assert np.array_equal(getattr(got, f), getattr(want, f)), f
        assert np.array_equal(fa.unpack(pk.tbuf), want.tbuf)
        with pytest.raises(N.NativeError) as e:
            K.collect_extension_jobs(None, l_pac - 1, reads, off, chains, seeds, ctx=ctx)
        assert e.value.code == N.FA_ERR_ARG
        ctx.set_reference(None)
        with pytest.raises(N.NativeError) as e:
            K.collect_extension_jobs(None, l_pac, reads, off, chains, seeds, ctx=ctx)
        assert e.value.code == N.FA_ERR_ARG
