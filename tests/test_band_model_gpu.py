"""Learned band predictor: GPU forward/backward against the NumPy restatement, model
file round trip, and learned-path results equal to the plain path's."""
import numpy as np
import pytest

import ferrousalign_b200 as fa
from ferrousalign_b200 import _native as N
from ferrousalign_b200 import band_model as B
from ferrousalign_b200 import synth
from oracle import band_mlp_oracle as M
from oracle import ksw_oracle as O

pytestmark = pytest.mark.gpu


def test_gradients_match_cpu_oracle(ctx):
    rng = np.random.default_rng(3)
    x = rng.normal(2.0, 3.0, size=(3000, 16)).astype(np.float32)
    t = rng.uniform(2.0, 6.5, size=3000).astype(np.float32)
    m = B.BandModel.create(seed=7)
    m.fit_norm(x)
    w, mu, sd = m.get()
    for tau in (0.5, 0.85):
        g, loss = m.grad(x, t, tau, ctx=ctx)
        gr, lr = M.grad(w, mu, sd, x, t, tau)
        assert abs(loss - lr) <= 1e-4 * max(1.0, abs(lr))
        # FP32 accumulation over 3000 samples against float64: relative 1e-3 of the largest entry
        assert np.max(np.abs(g - gr)) <= 1e-3 * np.max(np.abs(gr)) + 1e-6
    y, _ = m.predict(x[:500], ctx=ctx)
    _, _, _, yr = M.forward(w, mu, sd, x[:500])
    assert np.max(np.abs(y - yr)) <= 1e-4 * max(1.0, np.max(np.abs(yr)))


def test_features_match_restatement(ctx):
    b = synth.workload_ext_1m(3000, seed=406)
    b2 = synth.workload_ext_uneven(1000, seed=407, ref_len=2_000_000)
    p = fa.BandedPairWiseSW().to_struct()
    for batch in (b, b2):
        hints = B.hints_from_info(batch.info)
        x = B.features(p, batch.jobs, batch.qseq, batch.tseq, hints, ctx=ctx)
        xr = M.features(1, batch.jobs, batch.qseq, batch.tseq, hints)
        bad = np.argwhere(x != xr)
        assert len(bad) == 0, f"{len(bad)} feature values differ, first {bad[:3].tolist()}"
        assert len(np.unique(x[:, 14])) > 1 and len(np.unique(x[:, 15])) > 1


def test_first_band_rule(ctx):
    rng = np.random.default_rng(9)
    x = rng.normal(0.0, 1.0, size=(5000, 16)).astype(np.float32)
    w = rng.normal(0.0, 0.3, M.NPARAMS).astype(np.float32)
    w[M.O_B3] = 3.0                           # outputs spread over bands 1..2^9
    m = B.BandModel.create(seed=3)
    m.set(w=w, mean=x.mean(0), std=x.std(0))
    jobs = np.zeros(len(x), N.JOB_DT)
    jobs["w"] = rng.choice([20, 50, 100, 200], len(x))
    for margin, w_min in ((0.0, 2), (0.5, 4), (-0.3, 1)):
        y, band = m.predict(x, jobs=jobs, margin=margin, w_min=w_min, ctx=ctx)
        ref = M.first_band(y, margin, w_min, jobs["w"])
        e = np.clip(y.astype(np.float64) + margin, 0, 16)
        clear = np.abs(np.exp2(e) - np.round(np.exp2(e))) > 1e-3     # away from integer boundaries
        assert clear.mean() > 0.9
        assert np.array_equal(band[clear], ref[clear])


def test_training_reduces_loss_and_file_round_trip(ctx, tmp_path):
    rng = np.random.default_rng(5)
    x = rng.normal(0.0, 1.0, size=(20000, 16)).astype(np.float32)
    t = (3.0 + 0.8 * x[:, 0] - 0.5 * x[:, 3] + 0.3 * np.abs(x[:, 7])).astype(np.float32)
    m = B.BandModel.create(seed=1)
    m.fit_norm(x)
    losses = m.train(x, t, epochs=6, batch=2048, lr=3e-3, tau=0.5, ctx=ctx)
    assert losses[-1] < 0.5 * losses[0]
    p = tmp_path / "m.bin"
    m.save(p)
    m2 = B.BandModel.load(p)
    w1, mu1, sd1 = m.get()
    w2, mu2, sd2 = m2.get()
    assert np.array_equal(w1, w2) and np.array_equal(mu1, mu2) and np.array_equal(sd1, sd2)
    raw = bytearray(p.read_bytes())
    raw[200] ^= 0x40
    p.write_bytes(bytes(raw))
    with pytest.raises(N.NativeError):
        B.BandModel.load(p)


def test_learned_path_matches_plain_path(ctx):
    """Exact judge: results equal to the plain bwa-mem2 policy (proven by the exit-bound
    certificate), GPU decisions equal to the oracle's; fast judge: same decisions as the
    oracle (its equality with the plain path is empirical, so not asserted)."""
    b = synth.workload_ext_1m(30_000, seed=404)
    p = fa.BandedPairWiseSW().to_struct()
    plain, pst, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=fa.make_policy(N.FA_POLICY_BWA, 2), ctx=ctx)
    m = B.BandModel.load() if B.DEFAULT_MODEL.exists() else B.BandModel.create(seed=2)
    hints = B.hints_from_info(b.info)
    out, st, wf, wfin = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, m, hints=hints, ctx=ctx)
    assert np.array_equal(out, plain)
    ref, rwfin, _, rcells = O.ext_batch_policy(p, fa.make_policy(N.FA_POLICY_LEARNED, 2, B.JUDGE_LEARNED, 2), b.jobs,
                                               b.qseq, b.tseq, wf)
    assert np.array_equal(out, ref) and np.array_equal(wfin, rwfin)
    assert st["cells_executed"] == rcells.sum()
    out2, st2, wf2, _ = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, m, hints=hints, judge=B.JUDGE_FAST,
                                               w_min=16, ctx=ctx)
    ref2, _, _, _ = O.ext_batch_policy(p, fa.make_policy(N.FA_POLICY_LEARNED, 2, B.JUDGE_FAST, 16), b.jobs, b.qseq,
                                       b.tseq, wf2)
    assert np.array_equal(out2, ref2)


def test_network_beats_fixed_first_band(ctx):
    """What the trained network gains over the same policy without it: on a held-out
    batch every fixed first band executes more cells than the predicted first bands,
    all with results identical to the plain path."""
    if not B.DEFAULT_MODEL.exists():
        pytest.skip("no trained model file")
    b = synth.workload_ext_1m(200_000, seed=405)
    p = fa.BandedPairWiseSW().to_struct()
    plain, pst, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=fa.make_policy(N.FA_POLICY_BWA, 2), ctx=ctx)
    m = B.BandModel.load()
    out, st, _, _ = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, m, hints=B.hints_from_info(b.info), ctx=ctx)
    assert np.array_equal(out, plain)
    pol = fa.make_policy(N.FA_POLICY_LEARNED, 2, B.JUDGE_LEARNED, 1)
    for w0 in (2, 4, 8, 16, 32):
        o, s, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=pol,
                                  w_first=np.full(len(b.jobs), w0, np.int32), ctx=ctx)
        assert np.array_equal(o, plain)
        assert st["cells_executed"] < s["cells_executed"], f"fixed first band {w0} executes fewer cells"
    assert st["cells_executed"] * 2 < pst["cells_executed"]
