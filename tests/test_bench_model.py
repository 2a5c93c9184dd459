"""bench.py's algorithmic FLOP model (the roofline's numerator) against a
count of the reference algorithm's operations (src/lie_svd_small.rs)."""
import importlib.util
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def reference_flops(n, ns_iters, sweeps, rotations):
    # newton_schulz_polar (:158-183): per iteration X^T X and X (3I - X^T X), 2 n^3 each; the
    # final orthogonality check X^T X; solve (:296-323): Q^T A, Q V and the U^T U check
    products = (2 * ns_iters + 4) * 2 * n ** 3
    # eigh_jacobi_full (:212-285): per sweep the off-norm test over n(n-1)/2 entries (a
    # multiply and an add each); per rotation 2 rows/columns of A (n x 6) and 2 columns of V (n x 6)
    return products + sweeps * n * (n - 1) + rotations * 12 * n


def test_small_route_model_is_the_reference_count():
    b = _bench()
    rng = np.random.default_rng(0)
    n = rng.integers(5, 65, 200)
    it = rng.integers(5, 80, 200)
    sw = rng.integers(1, 15, 200)
    rot = rng.integers(0, 20000, 200)
    got = b.flops_per_matrix(n, it, sw, rot, np.ones(200, dtype=int))
    want = reference_flops(n.astype(float), it, sw, rot)
    assert np.allclose(got, want, rtol=0, atol=0)


def test_bss_model_counts_the_products_of_a_separation():
    # src/lie_svd_bss.rs:57-100: covariance, whitening and separation (2 C^2 T each), one lagged
    # covariance per kept lag (2 C^2 (T - lag)); the channel means and the centring update are
    # products with an inner dimension of 2 (4 C T each)
    b = _bench()
    ch, s = 32, 1000
    lags = [0, 1, 2, 3, 5, 1000, 2000]  # lag 0 and lags >= T are skipped
    want = 3 * 2 * ch * ch * s + sum(2 * ch * ch * (s - g) for g in (1, 2, 3, 5)) + 2 * 4 * ch * s
    assert b.bss_flops(ch, s, lags) == want
