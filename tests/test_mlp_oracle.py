"""CPU checks of the FP64 warm-start network restatement (oracle/mlp_oracle.py) that the GPU
gradient, Adam and inference tests compare against."""
import numpy as np

from oracle import mlp_oracle as M


def _case(n=37, seed=0):
    rng = np.random.default_rng(seed)
    p = (rng.normal(size=M.N_PARAMS) * 0.3).astype(np.float32)
    s = rng.uniform(0.5, 2.0, size=M.N_IN).astype(np.float32)
    x = rng.normal(size=(n, M.N_IN)).astype(np.float32)
    t = rng.normal(size=(n, M.N_OUT)).astype(np.float32)
    return p, s, x, t


def test_layout_size():
    assert M.N_PARAMS == 4866


def test_gradient_matches_central_differences():
    p, s, x, t = _case()
    p = p.astype(np.float64)
    _, g = M.loss_and_grad(p, s, x, t)
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.choice(np.arange(a, b), size=min(12, b - a), replace=False)
                          for a, b in [(M.W1, M.B1), (M.B1, M.W2), (M.W2, M.B2), (M.B2, M.W3), (M.W3, M.B3),
                                       (M.B3, M.N_PARAMS)]])
    eps = 1e-6
    for k in idx:
        d = np.zeros_like(p)
        d[k] = eps
        fd = (M.loss_and_grad(p + d, s, x, t)[0] - M.loss_and_grad(p - d, s, x, t)[0]) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])), (k, fd, g[k])


def test_loss_is_mean_of_summed_squares():
    p, s, x, t = _case()
    y = M.forward(p, s, x)
    assert np.isclose(M.loss_and_grad(p, s, x, t)[0], ((y - t) ** 2).sum() / x.shape[0])


def test_adam_first_step_is_signed_learning_rate():
    g = np.array([1e-3, -2.0, 0.0])
    p, m, v = M.adam(np.zeros(3), np.zeros(3), np.zeros(3), g, 0.01, 1)
    assert np.allclose(p, [-0.01, 0.01, 0.0], atol=1e-7)


def test_bf16_rounding_is_nearest_even():
    one = 1.0
    vals = np.array([one, one + 2.0 ** -9, one + 3 * 2.0 ** -9, -(one + 2.0 ** -8), 3.0e38])
    got = M._bf16(vals)
    # 1 + 2^-8 is half an ulp above 1: the tie goes to the even mantissa (1.0)
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == 1.0 + 2.0 ** -7 and got[3] == -1.0
    assert np.isfinite(got[4])


def test_init_layout():
    p = M.init_params(7)
    w1 = p[M.W1:M.B1].reshape(M.N_HID, M.N_IN)
    assert np.all(w1[:, 5:] == 0) and np.all(np.abs(w1[:, :5]) <= np.sqrt(1.2) + 1e-6)
    assert np.all(p[M.B1:M.W2] == 0) and np.all(p[M.B2:] == 0)
    assert np.abs(p[M.W2:M.B2]).max() <= np.sqrt(6 / 64) + 1e-6 and p[M.W2:M.B2].std() > 0.15
    assert not np.array_equal(p, M.init_params(8))
