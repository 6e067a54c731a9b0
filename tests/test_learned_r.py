"""Learned r predictor: feature function (CPU), gradient check of the CUDA
training kernels against a NumPy restatement, training progress, and that
the learned policy returns the same discords as the oracle (GPU)."""
import math

import numpy as np
import pytest

import paddi_b200 as P
from oracle import oracle as O
from paddi_b200 import datagen

F, H = 12, 64


# ------------------------------------------------------------ NumPy restatement
def _unpack(p):
    o = 0
    W1 = p[o:o + H * F].reshape(H, F); o += H * F
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


_erf = np.vectorize(math.erf)


def _gelu(z):
    return 0.5 * z * (1 + _erf(z / np.sqrt(2)))


def _gelu_d(z):
    return 0.5 * (1 + _erf(z / np.sqrt(2))) + z * np.exp(-0.5 * z * z) / np.sqrt(2 * np.pi)


def np_forward(p, X):
    W1, b1, W2, b2, W3, b3 = _unpack(p.astype(np.float64))
    z1 = X @ W1.T + b1
    h1 = _gelu(z1)
    z2 = h1 @ W2.T + b2
    h2 = _gelu(z2)
    return h2 @ W3 + b3, (z1, h1, z2, h2)


def np_grad(p, X, Y, tau):
    W1, b1, W2, b2, W3, b3 = _unpack(p.astype(np.float64))
    y, (z1, h1, z2, h2) = np_forward(p, X)
    e = Y - y
    loss = np.mean(np.where(e > 0, tau * e, (tau - 1) * e))
    dy = np.where(e > 0, -tau, 1 - tau) / len(Y)
    gW3 = h2.T @ dy
    gb3 = dy.sum()
    dz2 = (dy[:, None] * W3[None, :]) * _gelu_d(z2)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * _gelu_d(z1)
    gW1 = dz1.T @ X
    gb1 = dz1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return g, loss


def _data(n=300, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(0, 1, (n, F))
    Y = 0.3 * np.tanh(X[:, 0]) - 0.1 * X[:, 5] + 0.05 * rng.normal(size=n)
    return X.astype(np.float32), Y.astype(np.float32)


# ------------------------------------------------------------------ CPU tests
def test_numpy_gradient_matches_finite_differences():
    X, Y = _data(40)
    p = P.init_params(3).astype(np.float64)
    g, _ = np_grad(p, X.astype(np.float64), Y.astype(np.float64), 0.3)
    rng = np.random.default_rng(1)
    for i in rng.choice(len(p), 25, replace=False):
        h = 1e-6
        q1, q2 = p.copy(), p.copy()
        q1[i] += h
        q2[i] -= h
        l1 = np_grad(q1, X, Y, 0.3)[1]
        l2 = np_grad(q2, X, Y, 0.3)[1]
        assert g[i] == pytest.approx((l1 - l2) / (2 * h), rel=1e-3, abs=1e-7)


def test_feature_function():
    disc = [(100, 50.0), (101, 52.0), (101, 53.0), (99, 55.0), (102, 56.0), (102, 58.0)]
    f = P.r_features(disc, 6, 64, lb=57.0, flat_frac=0.25, prev_attempts=3)
    m = 70
    assert f[0] == pytest.approx(m / 1024)
    assert f[1] == pytest.approx(np.log(58.0 / (2 * m)), rel=1e-6)
    assert f[2] == pytest.approx(np.log(58.0 / 56.0), rel=1e-6)
    assert f[5] == pytest.approx(np.log(57.0 / 58.0), rel=1e-6)
    assert f[6] == 0.0 and f[7] == pytest.approx(0.2) and f[9] == pytest.approx(0.25)
    f0 = P.r_features([], 0, 64, 0.0, 0.0, 0)
    assert f0[0] == pytest.approx(64 / 1024) and not f0[1:9].any()


# ------------------------------------------------------------------ GPU tests
@pytest.mark.gpu
def test_cuda_gradient_matches_numpy():
    X, Y = _data(500)
    p = P.init_params(5)
    with P.Context() as c:
        g, loss = c.model_grad(X, Y, p, tau=0.2)
    gw, lw = np_grad(p.astype(np.float64), X.astype(np.float64), Y.astype(np.float64), 0.2)
    assert loss == pytest.approx(lw, rel=1e-4)
    np.testing.assert_allclose(g, gw, rtol=2e-3, atol=2e-6)


@pytest.mark.gpu
def test_cuda_forward_fp32_and_bf16():
    X, _ = _data(200)
    p = P.init_params(7)
    want, _ = np_forward(p, X.astype(np.float64))
    with P.Context() as c:
        y32 = c.model_predict(X, p, bf16=False)
        y16 = c.model_predict(X, p, bf16=True)
    np.testing.assert_allclose(y32, want, rtol=1e-4, atol=1e-5)
    assert np.max(np.abs(y16 - want)) < 0.05 * (np.max(np.abs(want)) + 1e-3)


@pytest.mark.gpu
def test_training_reduces_the_loss():
    X, Y = _data(4000, seed=2)
    with P.Context() as c:
        p, loss = c.model_train(X, Y, tau=0.2, epochs=60, batch=512, lr=3e-3, seed=1)
    assert loss[-1] < 0.5 * loss[0]
    # the pinball loss at tau puts about a fraction tau of the targets below
    with P.Context() as c:
        y = c.model_predict(X, p)
    assert 0.1 < np.mean(Y < y) < 0.35


@pytest.mark.gpu
def test_learned_policy_returns_the_same_discords_with_any_model():
    # an untrained model only changes the attempts, never the discords
    x, _ = datagen.palmad_series(n=8192, seed=5, n_anom=4, min_len=32, max_len=96)
    want, _ = O.palmad(x, 40, 56)
    for seed in (0, 1):
        with P.Context(r_policy=P.R_LEARNED, model=P.init_params(seed)) as c:
            got, log = c.palmad(x, 40, 56)
        assert [d.ind for d in got] == [w[0] for w in want]
        for d, w in zip(got, want):
            assert abs(d.dist - w[1]) <= 1e-5 * abs(w[1])
        assert any(e["r_source"] == 1 for e in log)


@pytest.mark.gpu
def test_trained_model_saves_attempts_on_held_out_series():
    """What the network gains: on held-out series of the evaluation recipe
    (seed 97, n = 2^20, lengths 64..1024; the model was trained on seed 31),
    the learned r policy takes fewer attempts than the exact bound alone and
    than the reference's MERLIN schedule, with identical discords."""
    from paddi_b200 import learned_r
    series = datagen.training_series(2, 1 << 20, 97, min_len=64, max_len=1024)
    rows = learned_r.evaluate(series, 64, 1024, model=learned_r.load_default())
    for r in rows:
        assert all(r[p] is not None and r[p]["same"] for p in r), r
        assert r["learned"]["attempts"] <= r["bound"]["attempts"], r
        assert r["learned"]["attempts"] < r["merlin"]["attempts"], r
    tot = {p: sum(r[p]["attempts"] for r in rows) for p in ("merlin", "bound", "learned")}
    assert tot["learned"] < tot["bound"] < tot["merlin"], tot
