"""The network oracle's gradient against central finite differences (FP64),
so that it can in turn check the GPU kernels."""
import numpy as np

from oracle import lmax_mlp as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(20, M.NF))
    T = rng.normal(size=20) * 0.5 + 5.0
    P = M.init(X, T, seed=1).astype(np.float64)

    # finite differences on the float64 function of the (unrounded) params:
    # evaluate with a float64 copy so that bf16 rounding does not hide steps
    def f(p):
        saved = M.bf16
        M.bf16 = lambda x: np.asarray(x, np.float64)
        try:
            return M.loss_and_grad(p, X, T)[0]
        finally:
            M.bf16 = saved

    saved = M.bf16
    M.bf16 = lambda x: np.asarray(x, np.float64)
    try:
        _, G, _ = M.loss_and_grad(P, X, T)
    finally:
        M.bf16 = saved
    for off in (M.OFF_W1 + 5, M.OFF_B1 + 3, M.OFF_W2 + 777, M.OFF_B2 + 9, M.OFF_W3 + 4000, M.OFF_B3 + 1,
                M.OFF_W4 + 17, M.OFF_B4):
        h = 1e-6
        pp, pm = P.copy(), P.copy()
        pp[off] += h
        pm[off] -= h
        fd = (f(pp) - f(pm)) / (2 * h)
        assert abs(fd - G[off]) <= 1e-5 * max(1.0, abs(fd)), (off, fd, G[off])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0            # halfway 1 + 2^-8 rounds to even
    assert r[2] == 1.0078125      # above halfway rounds up
    assert abs(r[3] + 3.140625) < 1e-12
