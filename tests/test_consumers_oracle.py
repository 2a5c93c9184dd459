"""The oracle's consumers (oracle/oracle_consumers.py) against the reference's
own tests of them: Phase-BSS (src/lie_svd_bss.rs:216-251) and the phase
normalizer's canonical wrappers (src/phase_normalizer.rs:377-413,
:1144-1229).  The reference's random draws come from StdRng, which is not
restated: the same constructions use numpy's generator, and the assertions
are the reference's (properties, not values)."""
import numpy as np

import oracle_consumers as OC


def bss_sources(channels=4, samples=512):
    # src/lie_svd_bss.rs:222-234
    t = np.arange(samples, dtype=np.float64)
    x = t / samples
    s = np.empty((channels, samples))
    for i in range(channels):
        if i == 0:
            s[i] = np.sin(2 * np.pi * 7.0 * x)
        elif i == 1:
            s[i] = np.sign(np.cos(2 * np.pi * 11.0 * x))
        elif i == 2:
            s[i] = np.sin(2 * np.pi * 3.0 * x) + 0.4 * np.sin(2 * np.pi * 17.0 * x)
        else:
            s[i] = np.sin((t * 37 + 11)) * 0.7
    i, j = np.meshgrid(np.arange(channels), np.arange(channels), indexing="ij")
    mixing = np.where(i == j, 1.0, 0.25 * np.sin((i * 13 + j * 7 + 3).astype(np.float64)))
    return s, mixing


def test_bss_improves_sir():
    s, mix = bss_sources()
    obs = mix @ s
    before = OC.estimate_sir_db(s, obs)
    r = OC.bss_separate(obs, OC.PhaseBssParams.for_channels(4))
    after = OC.estimate_sir_db(s, r.separated)
    assert after > before + 3.0, (before, after)
    assert r.trace.joint_final_offdiag <= r.trace.joint_initial_offdiag + 1e-10
    assert np.isfinite(r.trace.mean_channel_coherence)
    # unmixing applied to the centred observations gives the separated channels
    xc = OC.center_channels(obs)
    assert np.max(np.abs(r.unmixing @ xc - r.separated)) < 1e-10 * np.max(np.abs(r.separated))


def test_bss_lags_beyond_samples_fall_back_to_the_covariance():
    s, mix = bss_sources(3, 6)
    p = OC.PhaseBssParams.for_channels(3)
    p.lags = [0, 7]
    r = OC.bss_separate(mix @ s, p)
    assert r.separated.shape == (3, 6) and np.all(np.isfinite(r.separated))


def random_orthogonal(n, rng):
    q, _ = np.linalg.qr(rng.random((n, n)) - 0.5)
    return q


def test_canonical_scores_rotation_invariant_permutation_equivariant():
    rng = np.random.default_rng(1)
    a = rng.random((7, 5)) - 0.5
    sc = OC.canonical_row_scores(a)
    assert np.max(np.abs(OC.canonical_row_scores(a @ random_orthogonal(5, rng)) - sc)) < 1e-9
    perm = rng.permutation(7)
    assert np.max(np.abs(OC.canonical_row_scores(a[perm]) - sc[perm])) < 1e-9


def test_solve_canonicalized_invariant_to_row_and_column_order():
    rng = np.random.default_rng(101)
    n = 12
    base = rng.random((n, n)) - 0.5
    rp, cp = rng.permutation(n), rng.permutation(n)
    shuffled = base[np.ix_(rp, cp)]
    ub, sb, vb, _, _ = OC.solve_canonicalized(base)
    us, ss, vs, _, _ = OC.solve_canonicalized(shuffled)
    rec_b = (ub * sb) @ vb
    rec_s = (us[np.argsort(rp)] * ss) @ vs
    rec_s = rec_s[:, np.argsort(cp)]
    assert np.max(np.abs(rec_b - rec_s)) < 1e-8
    assert np.max(np.abs(rec_b - base)) < 1e-8


def test_diagonalize_symmetric_canonicalized_restores_the_basis():
    rng = np.random.default_rng(103)
    n = 6
    q = random_orthogonal(n, rng)
    fam = [q @ np.diag(1.0 + k * 0.4 + np.arange(n) * 0.2) @ q.T for k in range(3)]
    v, _, _, order = OC.diagonalize_symmetric_canonicalized(fam)
    for m in fam:
        r = v.T @ m @ v
        assert np.sum(np.abs(r - np.diag(np.diag(r)))) < 1e-6
    assert sorted(order) == list(range(n))
