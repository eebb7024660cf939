"""The region-merge kernel (csrc/region_kernel.cu) against the CPU restatement of
merge_scores_to_regions (oracle/region_oracle.py): random chains with edge values,
extension results from real extension batches, the device-resident entry and the
argument checks.  Bit-exact: every field of every region."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def random_chains(rng, n_chains, n_left, n_right, max_seeds=8):
    """Chains of 0-max_seeds seeds with positions that overlap (so coverage and ties
    happen), job indices that are absent (-1) or past the results now and then."""
    from ferrousalign_b200 import region as G
    counts = rng.integers(0, max_seeds + 1, n_chains)
    first = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    n = int(first[-1])
    seeds = np.zeros(n, G.SEED_EXT_DT)
    base = rng.integers(1 << 20, 1 << 40, n_chains).astype(np.uint64)
    qlen = rng.integers(40, 300, n_chains).astype(np.int32)
    ci = np.repeat(np.arange(n_chains), counts)
    seeds["query_pos"] = rng.integers(0, 40, n)
    seeds["query_pos"][rng.random(n) < 0.2] = 0
    seeds["len"] = rng.integers(5, 40, n)
    seeds["ref_pos"] = base[ci] + rng.integers(0, 60, n).astype(np.uint64)
    seeds["left_job"] = rng.integers(0, n_left, n)
    seeds["right_job"] = rng.integers(0, n_right, n)
    seeds["left_job"][rng.random(n) < 0.2] = -1
    seeds["right_job"][rng.random(n) < 0.2] = -1
    seeds["left_job"][rng.random(n) < 0.02] = n_left + 3     # ignored by the merge
    seeds["right_job"][rng.random(n) < 0.02] = n_right + 7
    return first, qlen, seeds


def random_results(rng, n):
    from ferrousalign_b200 import _native as N
    r = np.zeros(n, N.EXT_RESULT_DT)
    r["score"] = rng.integers(0, 200, n)
    r["qle"] = rng.integers(0, 150, n)
    r["tle"] = rng.integers(0, 200, n)
    r["gtle"] = rng.integers(0, 200, n)
    r["gscore"] = rng.integers(-1, 200, n)
    # gscore exactly at the clip threshold score - 5 and just above it
    k = rng.random(n)
    r["gscore"][k < 0.15] = r["score"][k < 0.15] - 5
    r["gscore"][(k >= 0.15) & (k < 0.3)] = r["score"][(k >= 0.15) & (k < 0.3)] - 4
    return r


def oracle_regions(opt, first, qlen, seeds, left, right):
    from oracle import region_oracle as R
    o = {k: int(opt[k][0]) for k in ("a", "pen_clip5", "pen_clip3", "w")}
    return R.merge_regions(o, first, qlen, seeds, left, right)


def test_random_chains_match_oracle(built):
    import ferrousalign_b200 as fa
    rng = np.random.default_rng(11)
    left, right = random_results(rng, 3000), random_results(rng, 2500)
    first, qlen, seeds = random_chains(rng, 6000, len(left), len(right))
    for opt in (fa.region_opts(), fa.region_opts(a=2, pen_clip5=0, pen_clip3=9, w=33)):
        out = fa.merge_scores_to_regions(first, qlen, seeds, left, right, opts=opt)
        ref = oracle_regions(opt, first, qlen, seeds, left, right)
        bad = np.nonzero(out != ref)[0]
        assert len(bad) == 0, (bad[:5], out[bad[:2]], ref[bad[:2]])
    assert (out["seed"] == -1).sum() > 0 and (out["seed"] >= 0).sum() > 5000


def test_regions_from_extension_batches(built):
    """Left and right jobs of the uneven workload through the extension kernels, their
    results merged per chain; the same chain table through the oracle's extension and
    merge gives the same regions."""
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import synth
    from oracle import ksw_oracle as O
    b = synth.workload_ext_uneven(20000)
    p = fa.BandedPairWiseSW().to_struct()
    lefts = np.nonzero(b.jobs["dir"] == 0)[0]
    rights = np.nonzero(b.jobs["dir"] == 1)[0]
    out, _, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq)
    ref_ext, _ = O.ext_batch(p, b.jobs, b.qseq, b.tseq)
    assert np.array_equal(out, ref_ext)
    rng = np.random.default_rng(5)
    first, qlen, seeds = random_chains(rng, 4000, len(lefts), len(rights), max_seeds=5)
    left_res, right_res = out[lefts], out[rights]
    got = fa.merge_scores_to_regions(first, qlen, seeds, left_res, right_res)
    want = oracle_regions(fa.region_opts(), first, qlen, seeds, ref_ext[lefts], ref_ext[rights])
    assert np.array_equal(got, want)


def test_device_entry_and_argument_checks(built):
    import torch
    import ferrousalign_b200 as fa
    from ferrousalign_b200 import _native as N
    lib = N.load()
    rng = np.random.default_rng(3)
    left, right = random_results(rng, 500), random_results(rng, 500)
    first, qlen, seeds = random_chains(rng, 900, len(left), len(right))
    opt = fa.region_opts()
    ref = oracle_regions(opt, first, qlen, seeds, left, right)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(a.view(np.uint8).copy()).to(dev)  # noqa: E731
    d_first, d_qlen, d_seeds, d_left, d_right = t(first), t(qlen), t(seeds), t(left), t(right)
    d_out = torch.zeros(len(qlen) * N.REGION_DT.itemsize, dtype=torch.uint8, device=dev)
    ctx = N.Context(0)
    N.check(lib.fa_merge_regions_device(ctx.handle, N.ptr(opt), d_first.data_ptr(), len(qlen), d_qlen.data_ptr(),
                                        d_seeds.data_ptr(), len(seeds), d_left.data_ptr(), len(left),
                                        d_right.data_ptr(), len(right), d_out.data_ptr(), None))
    N.check(lib.fa_ctx_sync(ctx.handle))
    got = d_out.cpu().numpy().view(N.REGION_DT)
    assert np.array_equal(got, ref)
    # result arrays only 4-byte aligned: the field-by-field loads, same regions
    pad = lambda a: torch.from_numpy(np.concatenate([np.zeros(4, np.uint8), a.view(np.uint8)])).to(dev)  # noqa: E731
    d_left4, d_right4 = pad(left), pad(right)
    d_out.zero_()
    N.check(lib.fa_merge_regions_device(ctx.handle, N.ptr(opt), d_first.data_ptr(), len(qlen), d_qlen.data_ptr(),
                                        d_seeds.data_ptr(), len(seeds), d_left4.data_ptr() + 4, len(left),
                                        d_right4.data_ptr() + 4, len(right), d_out.data_ptr(), None))
    N.check(lib.fa_ctx_sync(ctx.handle))
    assert np.array_equal(d_out.cpu().numpy().view(N.REGION_DT), ref)
    # a chain range past the seed array: reported by the kernel, no region for it
    bad_first = first.copy()
    bad_first[-1] = len(seeds) + 4
    d_bad = t(bad_first)
    N.check(lib.fa_merge_regions_device(ctx.handle, N.ptr(opt), d_bad.data_ptr(), len(qlen), d_qlen.data_ptr(),
                                        d_seeds.data_ptr(), len(seeds), d_left.data_ptr(), len(left),
                                        d_right.data_ptr(), len(right), d_out.data_ptr(), None))
    assert lib.fa_ctx_sync(ctx.handle) == N.FA_ERR_ARG
    assert d_out.cpu().numpy().view(N.REGION_DT)[-1]["seed"] == -1
    # host entry: ranges are checked before anything runs
    with pytest.raises(N.NativeError):
        fa.merge_scores_to_regions(bad_first, qlen, seeds, left, right)
    desc = first.copy()
    desc[1], desc[2] = desc[2], desc[1]
    if desc[1] != desc[2]:
        with pytest.raises(N.NativeError):
            fa.merge_scores_to_regions(desc, qlen, seeds, left, right)
    empty = fa.merge_scores_to_regions(np.zeros(1, np.uint32), np.zeros(0, np.int32), seeds, left, right)
    assert len(empty) == 0
    ctx.close()
