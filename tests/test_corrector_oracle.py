"""The CPU restatement of the learned corrector (oracle/corrector_ref.py) is
pinned by central finite differences of its own loss, in float64."""
import numpy as np

from oracle import corrector_ref as R


def test_corrector_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    feat = rng.standard_normal((2, 7, 9, R.CIN))
    target = rng.standard_normal((2, 7, 9))
    mask = (rng.uniform(size=(2, 7, 9)) > 0.2).astype(float)
    params = rng.standard_normal(R.NPARAM) * 0.3
    loss, grad, _ = R.loss_and_grad(feat, target, params, mask)
    idx = np.concatenate([rng.choice(R.N1, 12, replace=False),
                          R.N1 + rng.choice(R.N2, 12, replace=False),
                          R.N1 + R.N2 + rng.choice(R.N3, 8, replace=False)])
    h = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        fd = (R.loss_and_grad(feat, target, p1, mask)[0] - R.loss_and_grad(feat, target, p2, mask)[0]) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, grad[i])


def test_corrector_oracle_homogeneous_and_zero_params():
    rng = np.random.default_rng(1)
    feat = rng.standard_normal((1, 6, 8, R.CIN))
    params = rng.standard_normal(R.NPARAM) * 0.3
    y, _ = R.forward(feat, params)
    y2, _ = R.forward(3.5 * feat, params)
    assert np.allclose(y2, 3.5 * y, rtol=1e-12, atol=1e-12)  # bias-free ReLU net
    y0, _ = R.forward(feat, np.zeros(R.NPARAM))
    assert not np.any(y0)
