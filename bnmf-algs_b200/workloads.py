"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations of this path.

The reference publishes no datasets for bld_mult; its own benchmarks use
synthetic X (benchmark/bench_utils.hpp:24-33).  The generative model is the
allocation model of alloc_model::bnmf_priors / sample_S
(src/alloc_model/alloc_model_funcs.hpp:461-552): W columns ~ Dirichlet(alpha),
H ~ Dirichlet(beta), a Gamma scale, X ~ Poisson(scale * W H).  The Gamma is
drawn with b as a RATE (mean a/b), the parameterisation log_marginal_S uses
(alloc_model_funcs.hpp:145-169).
"""

import numpy as np


def _problem(X, z, a, b, alpha, beta, iters, name):
    return {"name": name, "X": np.ascontiguousarray(X, dtype=np.float64), "z": int(z),
            "a": float(a), "b": float(b),
            "alpha": np.ascontiguousarray(alpha, dtype=np.float64),
            "beta": np.ascontiguousarray(beta, dtype=np.float64), "iters": int(iters)}


def allocation_model_X(x, y, z, a, b, rng):
    """X ~ Poisson(scale * W H), W (x*z) columns ~ Dir(1), H (z*y) rows ~ Dir(1),
    scale ~ Gamma(shape a, rate b)."""
    W = rng.dirichlet(np.ones(x), size=z).T          # x*z, columns sum to 1
    H = rng.dirichlet(np.ones(y), size=z)            # z*y, rows sum to 1
    scale = rng.gamma(shape=a, scale=1.0 / b)
    return rng.poisson(scale * (W @ H)).astype(np.float64)


def plain_small(seed=0):
    """Plain FP64 bld_mult, CPU-runnable: x=64, y=48, z=8, 200 iterations."""
    rng = np.random.default_rng(seed)
    x, y, z = 64, 48, 8
    X = allocation_model_X(x, y, z, 5.0, 0.1, rng)
    return _problem(X, z, 5.0, 0.1, np.ones(x), np.ones(z), 200, "plain_64x48x8")


def plain_large(seed=1):
    """Single large plain solve: x=1024, y=1024, z=64 (67M-element S), 100 iterations."""
    rng = np.random.default_rng(seed)
    x, y, z = 1024, 1024, 64
    X = allocation_model_X(x, y, z, 5.0, 0.01, rng)
    return _problem(X, z, 5.0, 0.01, np.ones(x), np.ones(z), 100, "plain_1024x1024x64")


def zero_truncated_poisson(lam, rng):
    """Poisson(lam) conditioned on >= 1: draws of the entries that came out
    zero are repeated until they are not (exact rejection sampling; each
    entry keeps its own rate)."""
    lam = np.asarray(lam, dtype=np.float64)
    out = rng.poisson(lam).astype(np.float64)
    zero = np.flatnonzero(out == 0)
    flat_lam = lam.reshape(-1)
    flat = out.reshape(-1)
    while zero.size:
        draw = rng.poisson(flat_lam[zero])
        hit = draw > 0
        flat[zero[hit]] = draw[hit]
        zero = zero[~hit]
    return out


def precision_study(seed=2, x=2048, y=2048, z=32, zero_frac=0.3):
    """Heavy-tailed counts with ~30% exact zeros in total: per-row rates
    lambda_i ~ LogNormal(0, 1.5); each entry is a zero with probability
    zero_frac, otherwise a Poisson(lambda_i) count conditioned on >= 1 (a plain
    Poisson would add its own zeros, ~40% at these rates, on top of the
    mask).  alpha, beta ~ U(0.5, 2); 300 iterations."""
    rng = np.random.default_rng(seed)
    lam = rng.lognormal(0.0, 1.5, size=x)
    X = zero_truncated_poisson(lam[:, None] * np.ones((1, y)), rng)
    X[rng.random((x, y)) < zero_frac] = 0.0
    alpha = rng.uniform(0.5, 2.0, size=x)
    beta = rng.uniform(0.5, 2.0, size=z)
    return _problem(X, z, 5.0, 0.1, alpha, beta, 300, f"precision_{x}x{y}x{z}")


def batch_shapes(n=512, seed=3, lo=32, hi=512, zs=(4, 8, 16, 32, 64)):
    """(x, y, z) of the uneven batch: x, y log-uniform in [lo, hi], z uniform over zs."""
    rng = np.random.default_rng(seed)
    xs = np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), size=n))).astype(int)
    ys = np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), size=n))).astype(int)
    zz = rng.choice(np.array(zs), size=n)
    return [(int(a), int(b), int(c)) for a, b, c in zip(xs, ys, zz)]


def batch_instance(shape, seed):
    """One batch instance generated as in plain_small, with its own seed."""
    x, y, z = shape
    rng = np.random.default_rng(seed)
    X = allocation_model_X(x, y, z, 5.0, 0.1, rng)
    return _problem(X, z, 5.0, 0.1, np.ones(x), np.ones(z), 150, f"inst_{x}x{y}x{z}")


def batch(n=512, seed=3):
    return [batch_instance(s, 1000 + seed * 100003 + k) for k, s in enumerate(batch_shapes(n, seed))]


def serving_requests(n, rate_hz, seed=4, tail_frac=0.02, tail_shape=(4096, 4096, 32)):
    """Poisson arrival times (s) and shapes: the batch distribution plus a tail."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, size=n)
    times = np.cumsum(gaps) - gaps[0]
    shapes = batch_shapes(n, seed + 17)
    tail = rng.random(n) < tail_frac
    shapes = [tail_shape if t else s for s, t in zip(shapes, tail)]
    return times, shapes
