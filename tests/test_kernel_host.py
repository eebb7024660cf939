"""The int16x2 extension kernel's thread body, compiled for the host by nvcc, against
the oracle (no GPU needed).  This runs the exact kernel source, two jobs per thread,
including the segment logic that keeps the two jobs' band edges apart."""
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "kernel_host"))

import ferrousalign_b200 as fa  # noqa: E402
from ferrousalign_b200 import _native as N  # noqa: E402
from ferrousalign_b200 import synth  # noqa: E402
from oracle import ksw_oracle as O  # noqa: E402


@pytest.fixture(scope="module")
def host_lib(built):
    import build_host
    lib = C.CDLL(str(build_host.build()))
    lib.pair_host_run.restype = C.c_int
    lib.pair_host_run.argtypes = [C.c_void_p] * 3 + [C.c_uint32, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                                      C.c_void_p]
    return lib


def run_host(lib, p, jobs, qseq, tseq):
    """Longest-first order and 32-column capacity classes, as the library launches them."""
    q = jobs["qlen"]
    n = len(q)
    order = np.array(sorted(range(n), key=lambda i: (-int(q[i]), i)), np.uint32)
    out = np.zeros(n, N.EXT_RESULT_DT)
    st = np.zeros(1, np.uint32)
    s0 = 0
    while s0 < n:
        cap = (int(q[order[s0]]) + 31) // 32 * 32
        e0 = s0
        while e0 < n and q[order[e0]] > cap - 32:
            e0 += 1
        sub = np.ascontiguousarray(order[s0:e0])
        rc = lib.pair_host_run(p.ctypes.data, jobs.ctypes.data, sub.ctypes.data, len(sub), qseq.ctypes.data,
                               tseq.ctypes.data, int(q[order[s0]]), out.ctypes.data, st.ctypes.data)
        assert rc == 0
        s0 = e0
    return out, int(st[0])


def test_pairs_of_151bp_jobs(host_lib):
    b = synth.workload_ext_plain(3000)
    p = fa.BandedPairWiseSW().to_struct()
    out, st = run_host(host_lib, p, b.jobs, b.qseq, b.tseq)
    ref, _ = O.ext_batch(p, b.jobs, b.qseq, b.tseq)
    assert st == 0
    assert np.array_equal(out, ref), np.nonzero(out != ref)[0][:10]


@pytest.mark.parametrize("a,b_,n,gaps,w,zdrop", [(1, 4, -1, (6, 1, 6, 1), 100, 100), (2, 3, 0, (5, 2, 3, 1), 20, 30),
                                                 (3, 1, -1, (0, 1, 2, 2), 7, 0)])
def test_uneven_pairs_and_parameters(host_lib, a, b_, n, gaps, w, zdrop):
    ref_seq = synth.reference(400_000, seed=12, n_rate=0.02, repeat_frac=0.05)
    b = synth.ext_jobs(ref_seq, 1500, seed=19, read_len=(10, 160), seed_len=(3, 30), seed_at_start=False, w=w,
                       indel_rates=(0.0, 0.02, 0.06), sub_rate=0.04)
    sw = fa.BandedPairWiseSW(o_del=gaps[0], e_del=gaps[1], o_ins=gaps[2], e_ins=gaps[3], zdrop=zdrop,
                             mat=fa.bwa_fill_scmat(a, b_, n))
    p = sw.to_struct()
    out, st = run_host(host_lib, p, b.jobs, b.qseq, b.tseq)
    ref, _ = O.ext_batch(p, b.jobs, b.qseq, b.tseq)
    assert st == 0
    assert np.array_equal(out, ref), np.nonzero(out != ref)[0][:10]


def test_golden_cases_as_pairs(host_lib):
    """Every golden case with a bwa-form matrix, paired with the next such case."""
    cases = [c for c in json.loads((HERE / "golden" / "ext_cases.json").read_text())
             if c["mat"][0] in (1, 2, 3) and c["mat"][4] in (-1, 0) and all(
                 c["mat"][t * 5 + q] == (c["mat"][4] if 4 in (t, q) else (c["mat"][0] if t == q else c["mat"][1]))
                 for t in range(5) for q in range(5)) and (c["mat"][4] == 0 or c["mat"][1] <= -1)]
    assert len(cases) > 10
    for c0, c1 in zip(cases[::2], cases[1::2]):
        if any(c0[k] != c1[k] for k in ("mat", "o_del", "e_del", "o_ins", "e_ins", "zdrop", "end_bonus")):
            c1 = dict(c1, **{k: c0[k] for k in ("mat", "o_del", "e_del", "o_ins", "e_ins", "zdrop", "end_bonus")})
        p = np.zeros(1, N.PARAMS_DT)
        p["mat"][0] = np.array(c0["mat"], np.int8)
        p["m"] = 5
        for k in ("o_del", "e_del", "o_ins", "e_ins", "zdrop", "end_bonus"):
            p[k] = c0[k]
        qs = np.array(c0["query"] + c1["query"], np.uint8)
        ts = np.array(c0["target"] + c1["target"] + [0], np.uint8)
        jobs = np.zeros(2, N.JOB_DT)
        jobs[0] = (0, 0, len(c0["query"]), len(c0["target"]), c0["h0"], c0["w"], 1, 0)
        jobs[1] = (len(c0["query"]), len(c0["target"]), len(c1["query"]), len(c1["target"]), c1["h0"], c1["w"], 1, 0)
        out, st = run_host(host_lib, p, jobs, qs, ts)
        ref, _ = O.ext_batch(p, jobs, qs, ts)
        assert np.array_equal(out, ref), (c0["name"], c1["name"], out, ref)


# ---- two target rows per thread (extend_rows2_kernel.cu), same oracle


@pytest.fixture(scope="module")
def rows2_lib(built):
    import build_host
    lib = C.CDLL(str(build_host.build("rows2")))
    lib.rows2_host_run.restype = C.c_int
    lib.rows2_host_run.argtypes = ([C.c_void_p] * 3 + [C.c_uint32, C.c_void_p, C.c_void_p] + [C.c_int] * 3
                                   + [C.c_void_p] * 9)
    return lib


def run_rows2(lib, p, jobs, qseq, tseq, cert=0, ring=0, w_try=None, packed=None):
    """Longest-first order in 32-column capacity classes; returns results, per-job cells,
    status, the overflow jobs (the ones the kernel hands to the int32 kernel) and flags."""
    q = jobs["qlen"]
    n = len(q)
    order = np.array(sorted(range(n), key=lambda i: (-int(q[i]), i)), np.uint32)
    out = np.zeros(n, N.EXT_RESULT_DT)
    cells = np.zeros(n, np.uint32)
    flags = np.zeros(n, np.uint8)
    st = np.zeros(1, np.uint32)
    ovf = np.zeros(n, np.uint32)
    ovf_n = np.zeros(1, np.uint32)
    wt = None if w_try is None else np.ascontiguousarray(w_try, np.int32)
    ps = None if packed is None else [packed[0].struct(), packed[1].struct()]
    s0 = 0
    while s0 < n:
        cap = (int(q[order[s0]]) + 31) // 32 * 32
        e0 = s0
        while e0 < n and q[order[e0]] > cap - 32:
            e0 += 1
        sub = np.ascontiguousarray(order[s0:e0])
        rc = lib.rows2_host_run(p.ctypes.data, jobs.ctypes.data, sub.ctypes.data, len(sub), qseq.ctypes.data,
                                tseq.ctypes.data, int(q[order[s0]]), cert, ring,
                                None if wt is None else wt.ctypes.data, out.ctypes.data, flags.ctypes.data,
                                cells.ctypes.data, st.ctypes.data, ovf.ctypes.data, ovf_n.ctypes.data,
                                None if packed is None else ps[0].ctypes.data,
                                None if packed is None else ps[1].ctypes.data)
        assert rc == 0
        s0 = e0
    return out, cells, int(st[0]), np.sort(ovf[:int(ovf_n[0])]), flags


def check_rows2(lib, p, jobs, qseq, tseq, packed=None):
    out, cells, st, ovf, _ = run_rows2(lib, p, jobs, qseq, tseq, packed=packed)
    ref, tr = O.ext_batch(p, jobs, qseq, tseq)
    a = int(max(0, p["mat"][0].max()))
    wide = np.nonzero(jobs["h0"].astype(np.int64) + a * jobs["qlen"].astype(np.int64) > 255)[0]
    assert st == 0
    assert np.array_equal(ovf, wide.astype(np.uint32))
    keep = np.ones(len(jobs), bool)
    keep[wide] = False
    bad = np.nonzero(keep & (out != ref))[0]
    assert len(bad) == 0, (bad[:10], out[bad[:3]], ref[bad[:3]])
    assert np.array_equal(cells[keep], tr["cells"][keep].astype(np.uint32))
    return int(keep.sum())


def test_rows2_151bp_jobs(rows2_lib):
    b = synth.workload_ext_plain(3000)
    p = fa.BandedPairWiseSW().to_struct()
    assert check_rows2(rows2_lib, p, b.jobs, b.qseq, b.tseq) == 3000


@pytest.mark.parametrize("a,b_,n,gaps,w,zdrop", [(1, 4, -1, (6, 1, 6, 1), 100, 100), (2, 3, 0, (5, 2, 3, 1), 20, 30),
                                                 (3, 1, -1, (0, 1, 2, 2), 7, 0), (1, 2, -1, (3, 3, 1, 1), 3, 5),
                                                 (1, 4, 0, (6, 1, 6, 1), 1, 100)])
def test_rows2_uneven_jobs_and_parameters(rows2_lib, a, b_, n, gaps, w, zdrop):
    ref_seq = synth.reference(400_000, seed=12, n_rate=0.02, repeat_frac=0.05)
    b = synth.ext_jobs(ref_seq, 2000, seed=19, read_len=(10, 160), seed_len=(3, 30), seed_at_start=False, w=w,
                       indel_rates=(0.0, 0.02, 0.06), sub_rate=0.04)
    sw = fa.BandedPairWiseSW(o_del=gaps[0], e_del=gaps[1], o_ins=gaps[2], e_ins=gaps[3], zdrop=zdrop,
                             mat=fa.bwa_fill_scmat(a, b_, n))
    assert check_rows2(rows2_lib, sw.to_struct(), b.jobs, b.qseq, b.tseq) > 200


def test_rows2_golden_cases(rows2_lib):
    """Every golden case with a bwa-form matrix, one job at a time."""
    cases = [c for c in json.loads((HERE / "golden" / "ext_cases.json").read_text())
             if c["mat"][0] in (1, 2, 3) and c["mat"][4] in (-1, 0) and all(
                 c["mat"][t * 5 + q] == (c["mat"][4] if 4 in (t, q) else (c["mat"][0] if t == q else c["mat"][1]))
                 for t in range(5) for q in range(5)) and (c["mat"][4] == 0 or c["mat"][1] <= -1)]
    assert len(cases) > 10
    for c in cases:
        p = np.zeros(1, N.PARAMS_DT)
        p["mat"][0] = np.array(c["mat"], np.int8)
        p["m"] = 5
        for k in ("o_del", "e_del", "o_ins", "e_ins", "zdrop", "end_bonus"):
            p[k] = c[k]
        qs = np.array(c["query"], np.uint8)
        ts = np.array(c["target"] + [0], np.uint8)
        jobs = np.zeros(1, N.JOB_DT)
        jobs[0] = (0, 0, len(c["query"]), len(c["target"]), c["h0"], c["w"], 1, 0)
        if len(c["query"]) > 254:
            continue
        check_rows2(rows2_lib, p, jobs, qs, ts)


def check_rows2_cert(lib, p, jobs, qseq, tseq, w_try, ring):
    """Narrow runs at per-job bands w_try with the certificate: results and cells equal the
    oracle's run at that band, certificate bit and hint equal the oracle's trace (bit 1 =
    bound_ok and the configured band covers the first row's positive cells)."""
    jw = jobs.copy()
    jw["w"] = w_try
    out, cells, st, ovf, flags = run_rows2(lib, p, jobs, qseq, tseq, cert=1, ring=ring, w_try=w_try)
    ref, tr = O.ext_batch(p, jw, qseq, tseq)
    a = int(max(0, p["mat"][0].max()))
    wide = np.nonzero(jobs["h0"].astype(np.int64) + a * jobs["qlen"].astype(np.int64) > 255)[0]
    assert st == 0
    assert np.array_equal(ovf, wide.astype(np.uint32))
    keep = np.ones(len(jobs), bool)
    keep[wide] = False
    bad = np.nonzero(keep & (out != ref))[0]
    assert len(bad) == 0, (bad[:10], out[bad[:3]], ref[bad[:3]])
    assert np.array_equal(cells[keep], tr["cells"][keep].astype(np.uint32))
    clean = np.array([O.wide_clean(p, int(jobs["qlen"][k]), int(jobs["w"][k]), int(tr["init_reach"][k]))
                      for k in range(len(jobs))], bool)
    want_cert = (tr["bound_ok"] != 0) & clean
    want_hint = np.where(clean, tr["hint"], 63)
    assert np.array_equal((flags[keep] >> 1) & 1, want_cert[keep].astype(np.uint8)), \
        np.nonzero(((flags >> 1) & 1) != want_cert)[0][:10]
    assert np.array_equal(flags[keep] >> 2, want_hint[keep].astype(np.uint8))
    assert np.array_equal(flags[keep] & 1, (tr["clamped"][keep] != 0).astype(np.uint8))
    return int(keep.sum()), int(want_cert[keep].sum())


@pytest.mark.parametrize("ring", [0, 32, 64])
def test_rows2_certificate_matches_oracle(rows2_lib, ring):
    b = synth.workload_ext_1m(4000, seed=41)
    p = fa.BandedPairWiseSW().to_struct()
    rng = np.random.default_rng(ring + 1)
    cap = {0: 100, 32: 14, 64: 30}[ring]
    w_try = rng.integers(1, cap + 1, size=len(b.jobs)).astype(np.int32)
    n, ncert = check_rows2_cert(rows2_lib, p, b.jobs, b.qseq, b.tseq, w_try, ring)
    assert n == 4000 and 0 < ncert < n


@pytest.mark.parametrize("a,b_,n,gaps,zdrop", [(2, 3, 0, (5, 2, 3, 1), 30), (1, 2, -1, (3, 3, 1, 1), 5),
                                               (3, 1, -1, (0, 1, 2, 2), 0)])
def test_rows2_certificate_uneven_parameters(rows2_lib, a, b_, n, gaps, zdrop):
    ref_seq = synth.reference(400_000, seed=13, n_rate=0.02, repeat_frac=0.05)
    bt = synth.ext_jobs(ref_seq, 2000, seed=23, read_len=(10, 160), seed_len=(3, 30), seed_at_start=False, w=100,
                        indel_rates=(0.0, 0.02, 0.06), sub_rate=0.04)
    sw = fa.BandedPairWiseSW(o_del=gaps[0], e_del=gaps[1], o_ins=gaps[2], e_ins=gaps[3], zdrop=zdrop,
                             mat=fa.bwa_fill_scmat(a, b_, n))
    rng = np.random.default_rng(7)
    for ring, cap in ((0, 100), (32, 14), (64, 30)):
        w_try = rng.integers(1, cap + 1, size=len(bt.jobs)).astype(np.int32)
        check_rows2_cert(rows2_lib, sw.to_struct(), bt.jobs, bt.qseq, bt.tseq, w_try, ring)


# ---- job ordering (order_kernel.cu): the bin mapping shared by histogram and scatter


@pytest.fixture(scope="module")
def order_lib(built):
    import build_host
    lib = C.CDLL(str(build_host.build("order")))
    lib.order_host_bin.restype = C.c_int
    lib.order_host_bin.argtypes = [C.c_int]
    lib.order_host_run.restype = C.c_int
    lib.order_host_run.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    return lib


def test_order_bins_clamp_invalid_lengths(order_lib):
    """A live job with a negative query length lands in bin 0 (never bin -1, which would
    step a cursor before the histogram), an oversized one in the last bin."""
    assert order_lib.order_host_bin(-1) == 0
    assert order_lib.order_host_bin(-(2 ** 31)) == 0
    assert order_lib.order_host_bin(0) == 0
    assert order_lib.order_host_bin(151) == 151
    assert order_lib.order_host_bin(N.FA_MAX_QLEN) == N.FA_MAX_QLEN
    assert order_lib.order_host_bin(N.FA_MAX_QLEN + 1) == N.FA_MAX_QLEN
    assert order_lib.order_host_bin(2 ** 31 - 1) == N.FA_MAX_QLEN


def test_order_scatter_writes_every_slot_once(order_lib):
    rng = np.random.default_rng(5)
    q = rng.integers(1, 300, 5000).astype(np.int32)
    q[rng.choice(5000, 60, replace=False)] = rng.choice([-1, 0, -7, N.FA_MAX_QLEN + 5, -(2 ** 31)], 60)
    order = np.full(len(q), 0xFFFFFFFF, np.uint32)
    assert order_lib.order_host_run(q.ctypes.data, len(q), order.ctypes.data) == 0
    assert sorted(order.tolist()) == list(range(len(q)))
    b = np.clip(q[order], 0, N.FA_MAX_QLEN)
    assert np.all(b[:-1] >= b[1:])            # longest first


# ---- h0 = 0 under FA_PARAM_H0_ZERO: the kernels' closed form against the recurrence


def test_h0_zero_closed_form_matches_recurrence(rows2_lib, host_lib):
    """The oracle runs ksw_extend2's recurrence on h0 = 0 as written; the two-row kernel's
    thread body writes the closed form (all cells zero after row 0).  Same six fields and
    cell counts, over lengths and bands where row 0 does and does not reach the query end."""
    rng = np.random.default_rng(11)
    n = 400
    qlen = rng.integers(1, 200, n).astype(np.int32)
    tlen = rng.integers(0, 260, n).astype(np.int32)
    w = rng.integers(0, 150, n).astype(np.int32)
    qs = rng.integers(0, 5, int(qlen.sum())).astype(np.uint8)
    ts = rng.integers(0, 5, int(tlen.sum()) + 1).astype(np.uint8)
    jobs = np.zeros(n, N.JOB_DT)
    jobs["q_off"] = np.concatenate([[0], np.cumsum(qlen)[:-1]])
    jobs["t_off"] = np.concatenate([[0], np.cumsum(tlen)[:-1]])
    jobs["qlen"], jobs["tlen"], jobs["w"], jobs["dir"] = qlen, tlen, w, N.FA_DIR_RIGHT
    jobs["h0"] = np.where(rng.random(n) < 0.7, 0, rng.integers(1, 40, n))
    p = fa.BandedPairWiseSW(allow_h0_zero=True).to_struct()
    ref, tr = O.ext_batch(p, jobs, qs, ts)
    out, cells, st, ovf, flags = run_rows2(rows2_lib, p, jobs, qs, ts)
    assert st == 0 and len(ovf) == 0
    assert np.array_equal(out, ref), np.nonzero(out != ref)[0][:10]
    assert np.array_equal(cells.astype(np.int64), tr["cells"])
    pout, pst = run_host(host_lib, p, jobs, qs, ts)          # two jobs per thread
    assert pst == 0 and np.array_equal(pout, ref), np.nonzero(pout != ref)[0][:10]
    z = jobs["h0"] == 0
    assert np.all(out["score"][z] == 0) and np.all(out["max_off"][z] == 0)
    assert set(out["gscore"][z].tolist()) == {-1, 0}


def test_h0_zero_rejected_without_the_flag():
    p = fa.BandedPairWiseSW().to_struct()
    with pytest.raises(ValueError):
        O.ksw_extend2([0, 1, 2], [0, 1, 2], p["mat"][0], 6, 1, 6, 1, 100, 5, 100, 0)
    r, _ = O.ksw_extend2([0, 1, 2], [0, 1, 2], p["mat"][0], 6, 1, 6, 1, 100, 5, 100, 0, flags=N.FA_PARAM_H0_ZERO)
    assert (int(r["score"]), int(r["qle"]), int(r["tle"]), int(r["gtle"]), int(r["gscore"])) == (0, 0, 0, 1, 0)


# ---- 2-bit packed sequences: the same thread body reading packed bases and N runs


def test_pack_round_trip_and_runs():
    rng = np.random.default_rng(3)
    c = rng.integers(0, 4, 1001).astype(np.uint8)
    c[[0, 5, 6, 7, 500, 1000]] = 4
    ps = fa.pack(c)
    assert ps.n_bases == 1001 and len(ps.runs) == 4
    assert [tuple(int(x) for x in r) for r in ps.runs] == [(0, 1), (5, 3), (500, 1), (1000, 1)]
    assert np.array_equal(fa.unpack(ps), c)


@pytest.mark.parametrize("ring,cert", [(0, 0), (0, 1), (32, 1)])
def test_rows2_packed_reads_match_oracle(rows2_lib, ring, cert):
    """Uneven jobs with N-rich sequences (2% N, runs at job edges) through the two-row thread
    body reading 2-bit packed buffers: results, cells and certificate flags equal the byte-code
    run's and the oracle's."""
    ref_seq = synth.reference(400_000, seed=12, n_rate=0.02, repeat_frac=0.05)
    b = synth.ext_jobs(ref_seq, 1500, seed=23, read_len=(10, 160), seed_len=(3, 30), seed_at_start=False, w=20,
                       indel_rates=(0.0, 0.02, 0.06), sub_rate=0.04)
    p = fa.BandedPairWiseSW().to_struct()
    qp, tp = fa.pack(b.qseq), fa.pack(b.tseq)
    assert len(qp.runs) > 50 and len(tp.runs) > 50
    w_try = np.full(len(b.jobs), 12 if ring else 20, np.int32)
    got = run_rows2(rows2_lib, p, b.jobs, b.qseq, b.tseq, cert=cert, ring=ring, w_try=w_try, packed=(qp, tp))
    byt = run_rows2(rows2_lib, p, b.jobs, b.qseq, b.tseq, cert=cert, ring=ring, w_try=w_try)
    for a_, b_ in zip(got[:2] + got[3:], byt[:2] + byt[3:]):
        assert np.array_equal(a_, b_)
    assert got[2] == 0
    if not cert:
        check_rows2(rows2_lib, p, b.jobs, b.qseq, b.tseq, packed=(qp, tp))


@pytest.fixture(scope="module")
def packed_lib(built):
    import build_host
    lib = C.CDLL(str(build_host.build("packed")))
    lib.packed_host_read.restype = C.c_int
    lib.packed_host_read.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_void_p, C.c_void_p]
    return lib


@pytest.mark.parametrize("nw,r0,step", [(4, 0, 16), (7, -4, 16), (4, 8, 16), (2, 0, 8)])
def test_packed_span_reads_equal_four_base_reads(packed_lib, nw, r0, step):
    """The packed reader's multi-word spans (the band-feature windows, the query and target
    streams of the two-row kernel) give the bytes of the four-base reads and of the byte
    codes: N runs applied (runs at job edges, long and single), zero outside the job."""
    rng = np.random.default_rng(nw * 100 + r0)
    codes = rng.integers(0, 4, 60_000).astype(np.uint8)
    for _ in range(300):
        a = int(rng.integers(0, len(codes) - 40))
        codes[a:a + int(rng.integers(1, 40))] = 4
    codes[:3] = 4
    codes[-2:] = 4
    ps = fa.pack(codes)
    st = ps.struct()
    for off, ln in [(0, 151), (1, 77), (len(codes) - 151, 151), (len(codes) - 3, 3), (5, 0), (2, 1)] + \
            [(int(rng.integers(0, len(codes) - 300)), int(rng.integers(1, 300))) for _ in range(200)]:
        nsteps = max(1, (ln + step - 1) // step + 1)
        ow = np.zeros(nsteps * nw, np.uint32)
        o4 = np.zeros(nsteps * nw, np.uint32)
        assert packed_lib.packed_host_read(st.ctypes.data, off, ln, r0, step, nsteps, nw, ow.ctypes.data,
                                           o4.ctypes.data) == 0
        assert np.array_equal(ow, o4), (off, ln)
        pos = (r0 + np.arange(nsteps)[:, None] * step + np.arange(nw * 4)[None, :]).reshape(-1)
        ok = (pos >= 0) & (pos < ln)
        want = np.where(ok, codes[np.clip(off + pos, 0, len(codes) - 1)], 0).astype(np.uint8)
        assert np.array_equal(ow.view(np.uint8), want), (off, ln)


@pytest.mark.parametrize("h0_zero", [False, True])
@pytest.mark.parametrize("scoring", ["bwa", "a3"])
def test_rows2_int32_listing_matches_thread_body(rows2_lib, scoring, h0_zero):
    """The early overflow listing (rows2_int32_job, what rows2_ovf_list_kernel runs) selects
    exactly the jobs the two-row thread body hands on to the int32 kernel -- valid jobs on
    both sides of the 255 bound, and jobs its argument and capacity checks stop (h0 <= 0,
    qlen <= 0, tlen < 0, qlen past the capacity) -- so a two-row launch that skips the listed
    jobs plus an int32 pass over them runs every job exactly once."""
    lib = rows2_lib
    lib.rows2_host_int32_jobs.restype = None
    lib.rows2_host_int32_jobs.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p]
    sw = (fa.BandedPairWiseSW() if scoring == "bwa" else
          fa.BandedPairWiseSW(o_del=5, e_del=2, o_ins=3, e_ins=1, mat=fa.bwa_fill_scmat(3, 2, 0), zdrop=30))
    p = sw.to_struct()
    if h0_zero:
        p["flags"] = N.FA_PARAM_H0_ZERO
    a = int(p["mat"][0].max())
    rng = np.random.default_rng(91 + a)
    n, qcap = 3000, 200
    jobs = np.zeros(n, N.JOB_DT)
    jobs["qlen"] = rng.integers(-1, qcap + 12, n)
    jobs["tlen"] = rng.integers(-1, 240, n)
    jobs["h0"] = rng.choice(np.r_[np.arange(-1, 3), np.arange(230, 262), np.arange(3, 300, 7)], n)
    jobs["w"] = rng.integers(1, 24, n)
    jobs["q_off"] = rng.integers(0, 400, n)
    jobs["t_off"] = rng.integers(0, 400, n)
    # both sides of the bound: h0 + a * qlen == 255 and == 256
    k = np.arange(0, n, 5)
    ql = rng.integers(1, min(qcap, 250 // a) + 1, len(k))
    jobs["qlen"][k] = ql
    jobs["tlen"][k] = np.abs(jobs["tlen"][k])
    jobs["h0"][k] = 255 - a * ql + (np.arange(len(k)) & 1)
    qseq = rng.integers(0, 4, 1024).astype(np.uint8)
    tseq = rng.integers(0, 4, 1024).astype(np.uint8)
    order = np.arange(n, dtype=np.uint32)
    out = np.zeros(n, N.EXT_RESULT_DT)
    cells = np.zeros(n, np.uint32)
    flags = np.zeros(n, np.uint8)
    st = np.zeros(1, np.uint32)
    ovf = np.zeros(n, np.uint32)
    ovf_n = np.zeros(1, np.uint32)
    rc = lib.rows2_host_run(p.ctypes.data, jobs.ctypes.data, order.ctypes.data, n, qseq.ctypes.data,
                            tseq.ctypes.data, qcap, 0, 0, None, out.ctypes.data, flags.ctypes.data,
                            cells.ctypes.data, st.ctypes.data, ovf.ctypes.data, ovf_n.ctypes.data, None, None)
    assert rc == 0
    handed_on = np.sort(ovf[:int(ovf_n[0])])
    listed = np.zeros(n, np.uint8)
    lib.rows2_host_int32_jobs(p.ctypes.data, jobs.ctypes.data, n, qcap, listed.ctypes.data)
    assert np.array_equal(np.nonzero(listed)[0].astype(np.uint32), handed_on)
    assert 100 < len(handed_on) < n - 100
    assert listed[k[1::2]].all() and not listed[k[0::2]].any()


def test_rows2_skips_listed_jobs_with_a_null_list(rows2_lib):
    """With the overflow jobs listed ahead of the launch, the two-row thread body runs with a
    null list: it leaves exactly the listed jobs untouched (no result, no cells) and gives
    every other job the oracle's result."""
    lib = rows2_lib
    lib.rows2_host_int32_jobs.restype = None
    lib.rows2_host_int32_jobs.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_void_p]
    ref_seq = synth.reference(2_000_000, seed=8, n_rate=0.002, repeat_frac=0.05)
    b = synth.ext_jobs(ref_seq, 1500, seed=84, read_len=(40, 300), seed_at_start=False, seed_len=(10, 60))
    p = fa.BandedPairWiseSW().to_struct()
    jobs = b.jobs
    n = len(jobs)
    qcap = int(jobs["qlen"].max())
    order = np.arange(n, dtype=np.uint32)
    sentinel = np.array([(-7, -7, -7, -7, -7, -7)], N.EXT_RESULT_DT)[0]
    out = np.full(n, sentinel, N.EXT_RESULT_DT)
    cells = np.zeros(n, np.uint32)
    flags = np.zeros(n, np.uint8)
    st = np.zeros(1, np.uint32)
    rc = lib.rows2_host_run(p.ctypes.data, jobs.ctypes.data, order.ctypes.data, n, b.qseq.ctypes.data,
                            b.tseq.ctypes.data, qcap, 0, 0, None, out.ctypes.data, flags.ctypes.data,
                            cells.ctypes.data, st.ctypes.data, None, None, None, None)
    assert rc == 0 and int(st[0]) == 0
    listed = np.zeros(n, np.uint8)
    lib.rows2_host_int32_jobs(p.ctypes.data, jobs.ctypes.data, n, qcap, listed.ctypes.data)
    skip = listed.astype(bool)
    assert 10 < skip.sum() < n - 100
    assert (out[skip] == sentinel).all() and (cells[skip] == 0).all()
    ref, tr = O.ext_batch(p, jobs, b.qseq, b.tseq)
    bad = np.nonzero(~skip & (out != ref))[0]
    assert len(bad) == 0, (bad[:10], out[bad[:3]], ref[bad[:3]])
    assert np.array_equal(cells[~skip], tr["cells"][~skip].astype(np.uint32))
