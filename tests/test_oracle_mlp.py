"""The CPU oracle of the closure network (oracle/mlp.py), pinned by finite
differences: its backward pass is the derivative of its loss, to 1e-6 of
the gradient's scale, for weights and biases of every layer."""
import numpy as np

from oracle import mlp as M


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    dims = [20, 16, 16, 16, 6]
    W = [rng.standard_normal((dims[l], dims[l + 1])) / np.sqrt(dims[l]) for l in range(4)]
    B = [0.1 * rng.standard_normal(dims[l + 1]) for l in range(4)]
    x = rng.standard_normal((64, dims[0]))
    t = rng.standard_normal((64, dims[4]))
    nreal = 5
    _, grads = M.loss_and_grads(W, B, x, t, nreal)
    for l in range(4):
        gw, gb = grads[l]
        scale = max(np.abs(gw).max(), np.abs(gb).max())
        for _ in range(6):
            i, j = rng.integers(dims[l]), rng.integers(dims[l + 1])
            fd = M.fd_grad(W, B, x, t, nreal, l, (i, j))
            assert abs(fd - gw[i, j]) <= 1e-6 * scale, (l, i, j, fd, gw[i, j])
            fd = M.fd_grad(W, B, x, t, nreal, l, j, is_bias=True)
            assert abs(fd - gb[j]) <= 1e-6 * scale, (l, j, fd, gb[j])
    # the padded output columns carry no gradient
    assert np.all(grads[3][0][:, nreal:] == 0.0) and np.all(grads[3][1][nreal:] == 0.0)
