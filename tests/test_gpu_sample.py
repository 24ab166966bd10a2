"""GPU tests of the device data generation (bldm_bnmf_priors, bldm_sample_S,
bldm_sample_X), the allocation model's priors and sampler
(src/alloc_model/alloc_model_funcs.hpp:461-552).  The reference draws from
GSL's stream, which is not reproduced, so these check the distributions:
moments against their closed forms (at 5 standard errors), normalisation,
and determinism per seed."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(bldm, x, z, a=5.0, b=0.1, alpha=None, beta=None):
    return bldm.Params(a, b, np.ones(x) if alpha is None else alpha,
                       np.ones(z) if beta is None else beta)


def test_priors_normalised_and_deterministic(bldm):
    x, y, z = 60, 70, 6
    p = _params(bldm, x, z, alpha=np.linspace(0.5, 2.0, x), beta=np.linspace(0.3, 3.0, z))
    W, H, L = (t.cpu().numpy() for t in bldm.bnmf_priors((x, y, z), p, seed=3))
    assert W.shape == (x, z) and H.shape == (z, y) and L.shape == (y,)
    assert np.all(W >= 0) and np.all(H >= 0) and np.all(L > 0)
    np.testing.assert_allclose(W.sum(0), 1.0, atol=1e-12)
    np.testing.assert_allclose(H.sum(0), 1.0, atol=1e-12)
    W2, H2, L2 = (t.cpu().numpy() for t in bldm.bnmf_priors((x, y, z), p, seed=3))
    np.testing.assert_array_equal(W, W2)
    np.testing.assert_array_equal(L, L2)
    W3 = bldm.bnmf_priors((x, y, z), p, seed=4)[0].cpu().numpy()
    assert not np.array_equal(W, W3)


@pytest.mark.parametrize("a,b", [(5.0, 0.1), (0.5, 2.0), (40.0, 1.0)])
def test_gamma_moments(bldm, a, b):
    """L_j ~ Gamma(shape a, scale b): mean a b, variance a b^2 (a < 1 takes the boost)."""
    y = 200000
    L = bldm.bnmf_priors((2, y, 2), _params(bldm, 2, 2, a, b), seed=11)[2].cpu().numpy()
    mean, var = a * b, a * b * b
    assert abs(L.mean() - mean) <= 5 * np.sqrt(var / y)
    assert abs(L.var() - var) <= 0.05 * var


def test_dirichlet_moments(bldm):
    """W(:,k) ~ Dirichlet(alpha): component mean alpha_i / alpha_0."""
    x, z = 5, 100000
    alpha = np.array([0.5, 1.0, 2.0, 3.0, 0.2])
    W = bldm.bnmf_priors((x, 2, z), _params(bldm, x, z, alpha=alpha), seed=5)[0].cpu().numpy()
    a0 = alpha.sum()
    mean = alpha / a0
    var = alpha * (a0 - alpha) / (a0 * a0 * (a0 + 1))
    assert np.all(np.abs(W.mean(1) - mean) <= 5 * np.sqrt(var / z))


@pytest.mark.parametrize("mu", [0.03, 3.0, 25.0, 400.0])
def test_poisson_moments(bldm, mu):
    """S_ijk ~ Poisson(W_ik H_kj L_j) with a constant product mu (inversion below
    10, transformed rejection above): mean and variance mu, integer values."""
    import torch
    x, y, z = 200, 250, 8
    W = torch.full((x, z), 1.0 / x, dtype=torch.float64, device="cuda")
    H = torch.full((z, y), 1.0 / z, dtype=torch.float64, device="cuda")
    L = torch.full((y,), mu * x * z, dtype=torch.float64, device="cuda")
    S = bldm.sample_S(W, H, L, seed=7).cpu().numpy()
    n = S.size
    assert np.all(S == np.round(S)) and np.all(S >= 0)
    assert abs(S.mean() - mu) <= 5 * np.sqrt(mu / n)
    # the sample variance of n Poisson(mu) draws has variance (mu + 2 mu^2) / n
    assert abs(S.var() - mu) <= 5 * np.sqrt((mu + 2 * mu * mu) / n)
    S2 = bldm.sample_S(W, H, L, seed=7).cpu().numpy()
    np.testing.assert_array_equal(S, S2)


def test_sample_X_matches_summed_S(bldm):
    """X drawn directly has the mean of sum_k S_ijk; FP32 storage works alike."""
    import torch
    x, y, z = 300, 400, 8
    p = _params(bldm, x, z, a=5.0, b=40.0)
    W, H, L = bldm.bnmf_priors((x, y, z), p, seed=1)
    S = bldm.sample_S(W, H, L, seed=2)
    X = bldm.sample_X(W, H, L, seed=2)
    mu = (W @ H * L[None, :]).cpu().numpy()
    Xs = S.sum(2).cpu().numpy()
    Xd = X.cpu().numpy()
    assert abs(Xs.sum() - mu.sum()) <= 5 * np.sqrt(mu.sum())
    assert abs(Xd.sum() - mu.sum()) <= 5 * np.sqrt(mu.sum())
    W32, H32, L32 = bldm.bnmf_priors((x, y, z), p, seed=1, dtype=bldm.F32)
    X32 = bldm.sample_X(W32, H32, L32, seed=2)
    assert X32.dtype == torch.float32 and abs(float(X32.sum()) - mu.sum()) <= 5 * np.sqrt(mu.sum())


def test_priors_reject_bad_params(bldm):
    with pytest.raises(ValueError):
        bldm.bnmf_priors((4, 5, 3), _params(bldm, 3, 3))  # alpha size != x
    with pytest.raises(ValueError):
        bldm.bnmf_priors((4, 5, 3), _params(bldm, 4, 3, a=-1.0))
