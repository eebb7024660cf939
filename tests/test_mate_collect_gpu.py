"""The mate-rescue job kernels (csrc/mate_collect_kernel.cu) against the CPU restatement
of collect_rescue_jobs_for_read_soa (oracle/mate_collect_oracle.py): every job's read and
window bases, xtra word, attempt, orientation, strand, sequence and window; then the jobs
through the mate SW kernel against the oracle's ksw_align2.  Bit-exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rec_dict(x, dt):
    return {f: (rec_dict(x[f], dt[f]) if dt[f].names else int(x[f])) for f in dt.names}


def to_dicts(arr):
    return [rec_dict(x, arr.dtype) for x in arr]


def oracle_jobs(opts, bounds, pac, l_pac, chr_off, chr_len, reads, read_off, alns, cands):
    from oracle import mate_collect_oracle as M
    o = {k: int(opts[k][0]) for k in ("pen_unpaired", "max_matesw", "min_seed_len", "match_score")}
    rl = [list(reads[int(read_off[r]):int(read_off[r + 1])]) for r in range(len(read_off) - 1)]
    return M.collect(o, to_dicts(bounds), pac, l_pac, [int(x) for x in chr_off], [int(x) for x in chr_len], rl,
                     to_dicts(alns), to_dicts(cands))


def check(got, want):
    assert len(got.jobs) == len(want)
    for j, f, w in zip(got.jobs, got.info, want):
        assert {k: int(f[k]) for k in ("cand", "orientation", "is_rev", "rid", "adj_rb", "adj_re")} == \
            {k: w[k] for k in ("cand", "orientation", "is_rev", "rid", "adj_rb", "adj_re")}
        assert int(j["xtra"]) == w["xtra"]
        assert list(got.qbuf[int(j["q_off"]):int(j["q_off"]) + int(j["qlen"])]) == w["query"]
        assert list(got.tbuf[int(j["t_off"]):int(j["t_off"]) + int(j["tlen"])]) == w["target"]


def bounds_of(rows):
    from ferrousalign_b200 import _native as N
    b = np.zeros(4, N.INSERT_BOUNDS_DT)
    for k, (lo, hi, failed) in enumerate(rows):
        b[k] = (lo, hi, failed, 0)
    return b


def test_rescue_attempts_match_oracle(built):
    from ferrousalign_b200 import collect as K, mate_rescue as R, synth
    ref, chr_off, chr_len, reads, off, alns, cands = synth.workload_rescue(3000, ref_len=3_000_000)
    pac, l_pac = K.pack_reference(ref)
    for rows, opts in ((((0, 0, 1), (200, 600, 0), (0, 0, 1), (0, 0, 1)), R.rescue_opts()),
                       (((50, 900, 0), (150, 650, 0), (100, 1000, 0), (80, 300, 0)),
                        R.rescue_opts(pen_unpaired=40, max_matesw=1, min_seed_len=30)),
                       (((0, 0, 1), (200, 600, 0), (0, 0, 1), (0, 0, 1)), R.rescue_opts(max_matesw=-1))):
        bounds = bounds_of(rows)
        got = R.collect_rescue_jobs(pac, l_pac, chr_off, chr_len, reads, off, alns, cands, bounds, opts=opts)
        want = oracle_jobs(opts, bounds, pac, l_pac, chr_off, chr_len, reads, off, alns, cands)
        assert len(want) > 500
        check(got, want)


def test_rescue_jobs_through_mate_sw(built):
    from ferrousalign_b200 import collect as K, mate_rescue as R, synth
    from oracle import ksw_oracle as O
    ref, chr_off, chr_len, reads, off, alns, cands = synth.workload_rescue(1500, ref_len=3_000_000)
    pac, l_pac = K.pack_reference(ref)
    bounds = bounds_of(((0, 0, 1), (200, 600, 0), (0, 0, 1), (0, 0, 1)))
    got = R.collect_rescue_jobs(pac, l_pac, chr_off, chr_len, reads, off, alns, cands, bounds)
    mp = R.make_mate_params()
    out, _ = R.mate_sw_batch(mp, got.jobs, got.qbuf, got.tbuf)
    ref_out, _ = O.mate_batch(mp, got.jobs, got.qbuf, got.tbuf)
    assert np.array_equal(out, ref_out)
    # FR windows of true pairs contain the read: most rescues find it with a high score
    assert (out["score"] >= 100).mean() > 0.3


def test_argument_checks(built):
    from ferrousalign_b200 import _native as N, collect as K, mate_rescue as R, synth
    ref, chr_off, chr_len, reads, off, alns, cands = synth.workload_rescue(50, ref_len=500_000)
    pac, l_pac = K.pack_reference(ref)
    bounds = bounds_of(((0, 0, 1), (200, 600, 0), (0, 0, 1), (0, 0, 1)))
    bad = cands.copy()
    bad["anchor"]["ref_id"][0] = len(chr_off)
    with pytest.raises(N.NativeError):
        R.collect_rescue_jobs(pac, l_pac, chr_off, chr_len, reads, off, alns, bad, bounds)
    bad = cands.copy()
    bad["aln_first"][0] = len(alns)
    with pytest.raises(N.NativeError):
        R.collect_rescue_jobs(pac, l_pac, chr_off, chr_len, reads, off, alns, bad, bounds)
    with pytest.raises(N.NativeError):
        R.collect_rescue_jobs(pac, l_pac, chr_off, chr_len + np.uint64(l_pac), reads, off, alns, cands, bounds)


def test_resident_reference_and_reused_buffers(built):
    """The rescue collection reading the context's resident reference (pac=None) into reused
    page-locked HostBuffers equals the call that uploads the reference into fresh arrays."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import mate_rescue as R, synth
    ref, chr_off, chr_len, reads, off, alns, cands = synth.workload_rescue(1500, ref_len=3_000_000)
    pac, l_pac = fa.pack_reference(ref)
    bounds = bounds_of(((0, 0, 1), (200, 600, 0), (0, 0, 1), (0, 0, 1)))
    bufs = fa.HostBuffers()
    with fa.Context(0) as ctx:
        want = R.collect_rescue_jobs(pac, l_pac, chr_off, chr_len, reads, off, alns, cands, bounds, ctx=ctx)
        ctx.set_reference(pac, l_pac)
        for _ in range(2):
            got = R.collect_rescue_jobs(None, l_pac, chr_off, chr_len, reads, off, alns, cands, bounds, ctx=ctx,
                                        bufs=bufs)
            for f in ("jobs", "info", "qbuf", "tbuf"):
                assert np.array_equal(getattr(got, f), getattr(want, f)), f
