"""CPU tests of the correction-CNN oracle (oracle/cnn_oracle.py): its analytic
gradient against central finite differences in float64."""
import numpy as np

from oracle import cnn_oracle as CO


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, CO.N_PARAMS)
    x = rng.normal(0, 1, (2, 6, 7))
    t = rng.normal(0, 1, (2, 6, 7))
    loss, g = CO.loss_and_grads(p, x, t)
    idx = np.concatenate([rng.choice(np.arange(0, 144), 6), rng.choice(np.arange(144, 160), 3),
                          rng.choice(np.arange(160, 2464), 12), rng.choice(np.arange(2464, 2480), 3),
                          rng.choice(np.arange(2480, 2624), 6), [2624]])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (CO.loss_and_grads(pp, x, t)[0] - CO.loss_and_grads(pm, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_identity_at_zero_last_layer():
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.3, CO.N_PARAMS)
    p[2480:] = 0.0
    x = rng.normal(0, 1, (1, 5, 5))
    assert np.array_equal(CO.forward(p, x)["y"], x)
