"""The FP64 oracle of the learned-PME network (the checker of the BF16
training kernels) against central finite differences of its own loss."""
import numpy as np


def test_mlp_gradients_finite_difference(oracle):
    rng = np.random.default_rng(0)
    rows = 6
    x = rng.normal(size=(rows, 68))
    t = rng.normal(size=(rows, 3))
    p = rng.normal(scale=0.1, size=oracle.MLP_NPARAM)
    loss, g = oracle.mlp_grads(x, t, p)
    assert loss > 0
    # probe parameters in every block, including the last layer's bias
    offs = [0, 80 * 128 + 5, 80 * 128 + 128 + 300, oracle.MLP_NPARAM - 8 - 128 * 8 + 2 * 8 + 1,
            oracle.MLP_NPARAM - 8, oracle.MLP_NPARAM - 6]
    h = 1e-6
    for k in offs:
        q = p.copy()
        q[k] += h
        lp, _ = oracle.mlp_grads(x, t, q)
        q[k] -= 2 * h
        lm, _ = oracle.mlp_grads(x, t, q)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])
    # padded inputs (rows 68..79 of W1) and unused outputs (3..7) get no gradient
    W1 = g[: 80 * 128].reshape(80, 128)
    assert np.all(W1[68:] == 0)
    W4 = g[-8 - 128 * 8: -8].reshape(128, 8)
    assert np.all(W4[:, 3:] == 0) and np.all(g[-5:] == 0)
