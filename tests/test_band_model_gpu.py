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
    """Sound judge: results equal to the plain bwa-mem2 policy by construction; fast
    judge: equal on this batch (checked), with the cells it saves reported."""
    b = synth.workload_ext_1m(30_000, seed=404)
    p = fa.BandedPairWiseSW().to_struct()
    plain, pst, _ = fa.extend_batch(p, b.jobs, b.qseq, b.tseq, policy=fa.make_policy(N.FA_POLICY_BWA, 2), ctx=ctx)
    m = B.BandModel.load() if B.DEFAULT_MODEL.exists() else B.BandModel.create(seed=2)
    hints = B.hints_from_info(b.info)
    out, st, wf, wfin = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, m, hints=hints, judge=N.FA_JUDGE_CERT,
                                               ctx=ctx)
    assert np.array_equal(out, plain)
    # the oracle's learned policy with the same first bands agrees
    ref, rwfin, _, _ = O.ext_batch_policy(p, fa.make_policy(N.FA_POLICY_LEARNED, 2, N.FA_JUDGE_CERT, 4), b.jobs,
                                          b.qseq, b.tseq, wf)
    assert np.array_equal(out, ref) and np.array_equal(wfin, rwfin)
    out2, st2, wf2, _ = B.extend_batch_learned(p, b.jobs, b.qseq, b.tseq, m, hints=hints, judge=B.JUDGE_FAST, ctx=ctx)
    ref2, _, _, _ = O.ext_batch_policy(p, fa.make_policy(N.FA_POLICY_LEARNED, 2, B.JUDGE_FAST, 4), b.jobs, b.qseq,
                                       b.tseq, wf2)
    assert np.array_equal(out2, ref2)
    if B.DEFAULT_MODEL.exists():
        assert np.array_equal(out2, plain), f"{int((out2 != plain).sum())} of {len(plain)} differ"
        assert st2["cells_executed"] < pst["cells_executed"]
