"""Learned angular-order cutoff: the GPU kernels' gradient against the FP64
oracle, training on the GPU, and what the trained network gains over the
plain first range while leaving the cutoff and the outputs unchanged."""
import numpy as np
import pytest

import dsmsgt
from cases import psv_small
from dsmsgt import lmax_data
from oracle import lmax_mlp as M


@pytest.mark.gpu
def test_gradient_matches_oracle(built):
    rng = np.random.default_rng(0)
    X = rng.normal(size=(70, dsmsgt.LMAX_NFEAT)).astype(np.float32)
    T = (5.0 + 0.7 * np.tanh(X[:, 0]) + 0.2 * X[:, 1] ** 2).astype(np.float32)
    P = dsmsgt.lmax_init(X, T, seed=3)
    # biases away from zero so that their gradients are exercised
    P[M.OFF_B1:M.OFF_W2] = rng.normal(0, 0.1, M.H)
    G, loss = dsmsgt.lmax_grad(P, X, T)
    lref, Gref, _ = M.loss_and_grad(P, X, T)
    assert loss == pytest.approx(lref, rel=1e-4)
    for lo, hi in ((M.OFF_W1, M.OFF_B1), (M.OFF_B1, M.OFF_W2), (M.OFF_W2, M.OFF_B2), (M.OFF_B2, M.OFF_W3),
                   (M.OFF_W3, M.OFF_B3), (M.OFF_B3, M.OFF_W4), (M.OFF_W4, M.OFF_B4), (M.OFF_B4, M.NPARAM)):
        err = np.linalg.norm(G[lo:hi] - Gref[lo:hi]) / max(np.linalg.norm(Gref[lo:hi]), 1e-30)
        assert err <= 1e-4, (lo, hi, err)
    assert np.all(G[:M.OFF_W1] == 0.0)  # the standardisation is not trained


@pytest.mark.gpu
def test_training_fits_a_smooth_cutoff_law(built):
    rng = np.random.default_rng(1)
    X = rng.uniform(-1, 1, size=(2048, dsmsgt.LMAX_NFEAT)).astype(np.float32)
    T = (6.0 + 1.5 * X[:, 0] + 0.3 * X[:, 1] * X[:, 2] + 0.2 * np.sin(3 * X[:, 3])).astype(np.float32)
    P = dsmsgt.lmax_init(X, T, seed=0)
    P, losses = dsmsgt.lmax_train(X, T, P, epochs=150, batch=256, lr=2e-3)
    assert losses[-1] < 0.02 * losses[0], (losses[0], losses[-1])
    _, _, pred = M.loss_and_grad(P, X[:256], T[:256])
    assert np.median(np.abs(pred - T[:256])) < 0.05


def harvest_small(seeds, imax, freqs, r0s=(6071.0, 5771.0)):
    X, T = [], []
    for sd in seeds:
        for r0 in r0s:
            s = dsmsgt.Setup(psv_small(seed=sd, imax=imax, r0=r0), "psv")
            ctx = dsmsgt.Context(s)
            ll = ctx.cutoffs(freqs)
            f = ctx.lmax_features(freqs)
            X.append(f)
            T.append((np.log(ll) - f[:, 0]).astype(np.float32))  # relative to the lsuf scale
            ctx.close()
    return np.concatenate(X), np.concatenate(T)


@pytest.mark.gpu
def test_cutoffs_only_equal_full_run(built):
    s = dsmsgt.Setup(psv_small(), "psv")
    ctx = dsmsgt.Context(s)
    fr = [1, 17, 50]
    ll = ctx.cutoffs(fr)
    _, _, _, llf = ctx.run(fr)
    ctx.close()
    assert list(ll) == list(llf)


@pytest.mark.gpu
def test_learned_ranges_gain_without_changing_results(built):
    """Trained on six seeded models, evaluated on a seventh: the learned first
    ranges solve fewer systems, and the cutoffs and every output equal the
    plain method's.  At low frequencies the amplitude test stops far above
    lsuf, where the plain first range (max(512, lsuf + 64)) needs extra
    rounds; the network predicts those cutoffs."""
    imax = 256
    train_freqs = list(range(1, imax + 1, 8))
    X, T = harvest_small([1, 2, 3, 4, 5, 6], imax, train_freqs)
    P = dsmsgt.lmax_init(X, T, seed=0)
    P, losses = dsmsgt.lmax_train(X, T, P, epochs=300, batch=64, lr=2e-3)
    s = dsmsgt.Setup(psv_small(seed=0, imax=imax), "psv")
    fr = list(range(3, imax + 1, 16))
    plain = dsmsgt.Context(s, freq_batch=8)
    t0, r0, y0, l0 = plain.run(fr)
    st0 = plain.stats()
    plain.close()
    learned = dsmsgt.Context(s, freq_batch=8, use_lmax_predictor=1)
    learned.set_lmax_model(P)
    t1, r1, y1, l1 = learned.run(fr)
    st1 = learned.stats()
    pl = learned.lmax_predict(fr)
    learned.close()
    # same truncation and the same numbers: only the padded solves differ
    assert list(l0) == list(l1)
    assert np.array_equal(t0, t1) and np.array_equal(r0, r1) and np.array_equal(y0, y1)
    miss = float(np.mean(np.exp(pl) * lmax_data.MARGIN + lmax_data.PAD < l0))
    print(f"systems plain {st0.systems} learned {st1.systems}; padded orders {st0.orders_padded} -> "
          f"{st1.orders_padded}; miss rate {miss:.3f}; final loss {losses[-1]:.4f}")
    assert st1.systems < st0.systems
    assert st1.orders_padded < st0.orders_padded
