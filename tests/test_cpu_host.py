"""Host-side checks that need no GPU: the C ABI library loads and exports every
symbol the header declares, struct layouts agree, the generator is deterministic and
the oracle's batch drivers and retry policy behave."""
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    text = (ROOT / "include" / "ferrous_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fa_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol(built):
    import ferrousalign_b200._native as N
    lib = N.load()
    names = header_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(N.SIGNATURES), "ctypes signatures must cover exactly the header"


def test_mate_xtra_matches_reference_formula(built):
    import ferrousalign_b200._native as N
    lib = N.load()
    # mate_rescue.rs:314-321: XSUBO|XSTART|(XBYTE if len*a<250)|min_seed_len*a
    assert lib.fa_mate_xtra(151, 1, 19) == (0x40000 | 0x80000 | 0x10000 | 19)
    assert lib.fa_mate_xtra(300, 1, 19) == (0x40000 | 0x80000 | 19)
    from ferrousalign_b200 import mate_xtra
    assert mate_xtra(151, 1, 19) == lib.fa_mate_xtra(151, 1, 19)


def test_struct_sizes_match_header(built):
    import ctypes as C
    import ferrousalign_b200._native as N
    # compile-free check: offsets of the packed records used across the ABI
    assert N.JOB_DT.fields["qlen"][1] == 16 and N.JOB_DT.fields["dir"][1] == 32
    assert N.PARAMS_DT.fields["m"][1] == 28
    assert N.STATS_DT.fields["kernel_ms"][1] == 32
    assert C.sizeof(C.c_void_p) == 8


def test_synth_deterministic(built):
    from ferrousalign_b200 import synth
    a = synth.workload_ext_plain(2000)
    b = synth.workload_ext_plain(2000)
    assert np.array_equal(a.jobs, b.jobs) and np.array_equal(a.qseq, b.qseq) and np.array_equal(a.tseq, b.tseq)
    j = a.jobs
    assert (j["qlen"] == 151 - a.info["seed_len"]).all()
    assert (j["h0"] == a.info["seed_len"]).all()
    assert (j["tlen"] == j["qlen"] + 100).all()
    assert a.qseq.max() <= 4 and a.tseq.max() <= 4
    # thread count does not change the output
    ref = synth.reference(1_000_000, seed=1, n_rate=0.001)
    c = synth.ext_jobs(ref, 500, seed=101, threads=1)
    d = synth.ext_jobs(ref, 500, seed=101, threads=7)
    assert np.array_equal(c.jobs, d.jobs) and np.array_equal(c.tseq, d.tseq)


def test_synth_uneven_and_mate(built):
    from ferrousalign_b200 import synth
    ref = synth.reference(2_000_000, seed=3, n_rate=0.001, repeat_frac=0.05)
    b = synth.ext_jobs(ref, 3000, seed=9, read_len=(50, 300), seed_at_start=False)
    assert set(np.unique(b.jobs["dir"])) == {0, 1}
    assert b.jobs["qlen"].max() <= 300
    m = synth.mate_jobs(ref, 200, seed=4)
    assert (m.jobs["qlen"] == 151).all() and (m.jobs["tlen"] == 551).all()


def test_oracle_batch_matches_single(built):
    from ferrousalign_b200 import BandedPairWiseSW, synth
    from oracle import ksw_oracle as O
    b = synth.workload_ext_plain(300)
    p = BandedPairWiseSW().to_struct()
    out, tr = O.ext_batch(p, b.jobs, b.qseq, b.tseq, threads=3)
    for i in range(0, 300, 37):
        j = b.jobs[i]
        qo, to = int(j["q_off"]), int(j["t_off"])
        q = b.qseq[qo:qo + int(j["qlen"])]
        t = b.tseq[to:to + int(j["tlen"])]
        r, t1 = O.ksw_extend2(q, t, p["mat"][0], 6, 1, 6, 1, int(j["w"]), 5, 100, int(j["h0"]))
        assert tuple(r) == tuple(out[i]) and t1["cells"] == tr[i]["cells"]


def test_oracle_policy_certificate_is_exact(built):
    """A narrow run whose band clamp never bound equals the run at the full band."""
    from ferrousalign_b200 import BandedPairWiseSW, make_policy, synth
    from oracle import ksw_oracle as O
    ref = synth.reference(200_000, seed=5, n_rate=0.0)
    b = synth.ext_jobs(ref, 400, seed=3, read_len=(40, 60), seed_len=(30, 35), sub_rate=0.0,
                       indel_rates=(0.0,))
    p = BandedPairWiseSW(zdrop=20).to_struct()
    plain, _, _, _ = O.ext_batch_policy(p, make_policy(1, 2), b.jobs, b.qseq, b.tseq)
    wf = np.full(len(b.jobs), 4, np.int32)
    learned, wfin, tries, _ = O.ext_batch_policy(p, make_policy(2, 2, 1, 1), b.jobs, b.qseq, b.tseq, wf)
    assert np.array_equal(plain, learned)


def test_host_buffers_reuse_and_grow():
    """HostBuffers hands out views of one storage per name: reused while a request fits,
    replaced by a larger one when it does not; dtypes and shapes as asked."""
    from ferrousalign_b200.hostbuf import HostBuffers, out_array
    b = HostBuffers(pinned=False)
    a = b.get("x", 100, np.uint32)
    a[:] = 7
    c = b.get("x", 50, np.uint32)
    assert c.shape == (50,) and c.dtype == np.uint32 and np.shares_memory(a, c) and (c == 7).all()
    d = b.get("x", 400, np.uint64)
    assert d.shape == (400,) and not np.shares_memory(a, d)
    e = b.get("y", 3, np.dtype([("a", "<u4"), ("b", "<u8")]))
    assert e.shape == (3,) and not np.shares_memory(d, e)
    assert (out_array(None, "z", 5, np.int32, zero=True) == 0).all()
    assert out_array(b, "x", 10, np.uint64).base is not None
