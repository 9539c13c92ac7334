"""The scheduler MLP's CPU oracle: analytic gradient = central differences."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
import mlp_oracle as M  # noqa: E402


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, M.NPARAM)
    x = rng.normal(0, 1, (17, M.IN))
    t = rng.normal(0, 1, (17, M.OUT))
    loss, g = M.loss_and_grad(p, x, t)
    gn = M.numeric_grad(p, x, t)
    assert loss > 0
    np.testing.assert_allclose(g, gn, rtol=1e-5, atol=1e-8)
