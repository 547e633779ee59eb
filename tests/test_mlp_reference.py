"""The numpy restatement of the surrogate network (the CPU reference for the tensor-core kernels)
checked against central finite differences of its own loss."""
import numpy as np

from tests.mlp_reference import loss_and_grads


def test_reference_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    dims = [(7, 5), (7, 7), (4, 7)]
    params = [(rng.standard_normal(d) * 0.5, rng.standard_normal(d[0]) * 0.1) for d in dims]
    X = rng.standard_normal((13, 5))
    T = rng.standard_normal((13, 4))
    _, grads = loss_and_grads(params, X, T)
    h = 1e-6
    for l, (W, b) in enumerate(params):
        for arr, g in ((W, grads[l][0]), (b, grads[l][1])):
            flat = arr.reshape(-1)
            for k in rng.choice(flat.size, size=min(6, flat.size), replace=False):
                old = flat[k]
                flat[k] = old + h
                lp, _ = loss_and_grads(params, X, T)
                flat[k] = old - h
                lm, _ = loss_and_grads(params, X, T)
                flat[k] = old
                assert abs((lp - lm) / (2 * h) - g.reshape(-1)[k]) <= 1e-6 * max(1.0, abs(g.reshape(-1)[k]))
