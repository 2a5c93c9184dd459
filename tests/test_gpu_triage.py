"""GPU triage (lsvd_triage_batched_f64) against the oracle's restatement of
analyze_matrix / choose_route (src/lie_svd_adaptive.rs:84-274),
phase_signature (src/lie_svd_phasehealth.rs:100-343) and the PhaseEngine
passport (src/lie_svd_engine.rs:75-103), plus the reference's routing and
PhaseEngine tests through the GPU.

Bars: every statistic within 1e-12 absolute + 1e-11 relative of the oracle's
(the same sums in a different order; atan2/log/sin/cos from CUDA), routes
identical."""
import numpy as np
import pytest

import oracle as O
from lie_cliffalg_analog_svd_b200 import LieSvdAdaptive, PhaseEngine, triage_batched
from lie_cliffalg_analog_svd_b200 import _lib as L
from lie_cliffalg_analog_svd_b200 import profiles as P
from lie_cliffalg_analog_svd_b200.api import _triage_dict

pytestmark = pytest.mark.gpu


def upper_shift(n, d=1.0, u=3.0):
    return np.diag(np.full(n, d)) + np.diag(np.full(n - 1, u), 1)


def _cases():
    rng = np.random.default_rng(3)
    i, j = np.meshgrid(np.arange(24), np.arange(24), indexing="ij")
    r9, c14 = np.meshgrid(np.arange(9), np.arange(14), indexing="ij")
    return [rng.standard_normal((n, n)) for n in (1, 2, 4, 5, 16, 33, 64, 200, 700)] + [
        np.where(i // 6 == j // 6, 4.0, 0.02) + np.sin(((i + j) * 31).astype(float)) * 1e-3,
        np.sin((i * 13 + j * 7 + 3).astype(float)), upper_shift(12), upper_shift(24, 1.0, 5.0),
        upper_shift(128, 1.0, 5.0), np.diag([4.0, 3.0, 2.0, 1.0, 0.5, 0.25]), np.zeros((8, 8)),
        np.sin((r9 * 7 + c14 * 11 + 3).astype(float)), rng.standard_normal((30, 7)), rng.standard_normal((3, 50)),
        rng.standard_normal((64, 64)) + rng.standard_normal((64, 64)).T]


def test_triage_matches_oracle():
    mats = _cases()
    out = triage_batched(mats)
    for a, rec in zip(mats, out):
        g, o = _triage_dict(rec), O.triage(a)
        assert g["route"] == o["route"] and g["passport_route"] == o["passport_route"], (a.shape, g, o)
        for f in L.TRIAGE_FIELDS:
            x, y = g[f], o[f]
            if np.isnan(y):
                assert np.isnan(x), (a.shape, f)
            else:
                assert abs(x - y) <= 1e-12 + 1e-11 * abs(y), (a.shape, f, x, y)


def test_reference_routing_through_gpu():  # src/lie_svd_adaptive.rs:395-552
    n = 16
    assert LieSvdAdaptive.choose_route(np.diag(2.0 - np.arange(n) / n)) == "Small"
    i, j = np.meshgrid(np.arange(24), np.arange(24), indexing="ij")
    stress = np.where(i // 6 == j // 6, 4.0, 0.02) + np.sin(((i + j) * 31).astype(float)) * 1e-3
    assert LieSvdAdaptive.choose_route(stress) == "CoreFlowTopo"
    assert LieSvdAdaptive.choose_route(np.sin((i * 13 + j * 7 + 3).astype(float))) == "Small"
    assert LieSvdAdaptive.choose_route(upper_shift(24, 1.0, 5.0)) == "PhaseFlow"
    assert LieSvdAdaptive.choose_route(upper_shift(128, 1.0, 5.0)) == "Small"
    with pytest.raises(L.LsvdError):
        LieSvdAdaptive.analyze_matrix(np.ones((3, 4)))


def test_adaptive_solve_with_trace():  # src/lie_svd_adaptive.rs:83-100
    # Small and Micro routes run as the reference runs them; a PhaseFlow route is
    # reported and solved by the exact tier, to the same bars
    for a, route, taken in ((np.diag(2.0 - np.arange(16) / 16), "Small", "Small"),
                            (np.array([[3.0, 1.0], [0.5, 2.0]]), "Micro", "Micro"),
                            (upper_shift(24, 1.0, 5.0), "PhaseFlow", "Small")):
        (u, s, vt), tr = LieSvdAdaptive.solve_with_trace(a)
        assert (tr["route"], tr["route_taken"]) == (route, taken)
        assert tr["triage"]["route"] == route
        so = (O.LieSvdMicro if a.shape[0] <= 4 else O.LieSvdSmall).solve(a)[1]
        assert np.max(np.abs(s - so)) <= 1e-13 * so.max()
        assert np.linalg.norm((u * s) @ vt - a) <= 4e-13 * np.linalg.norm(a)
    u, s, vt = LieSvdAdaptive.solve(np.diag(2.0 - np.arange(16) / 16))
    assert np.allclose(np.sort(s), np.sort(2.0 - np.arange(16) / 16), atol=1e-14)
    with pytest.raises(L.LsvdError):
        LieSvdAdaptive.solve_with_trace(np.eye(4), params={"small_max_n": 10})


def test_batched_workload_routes():
    # the benchmark's uneven batch: every matrix gets its route on the device
    ns, a, _ = P.uneven_batch_workload(3000, seed=8)
    ao = np.concatenate([[0], np.cumsum(ns.astype(np.int64) ** 2)])
    mats = [a[ao[t]:ao[t + 1]].reshape(n, n) for t, n in enumerate(ns)]
    out = triage_batched(mats)
    for t in range(0, len(mats), 37):
        o = O.triage(mats[t])
        assert O.ADAPTIVE_ROUTES[out["adaptive_route"][t]] == o["route"]
        assert abs(out["offdiag_ratio"][t] - o["offdiag_ratio"]) <= 1e-12
    assert np.all(out["adaptive_route"][ns <= 4] == 0)


def test_phase_engine_facade():  # src/lie_svd_engine.rs:338-362
    (u, s, vt), rep = PhaseEngine.solve_real(np.eye(6))
    assert rep.passport["rows"] == 6 and rep.rel_recon < 1e-12
    # the identity's rows all twist (ratio 1): the reference routes it to PhaseFlow,
    # which this library replaces by the exact route
    assert rep.passport["route_hint"] == "RealPhaseFlowPolished" and rep.route == "RealSmall"
    pp = PhaseEngine.passport_real(upper_shift(8))
    assert np.isfinite(pp["global_phase"]) and pp["torsion_energy"] > 0
    assert 0 <= pp["chirality_balance"] <= 1 and 0 <= pp["phase_entropy"] <= 1
    # a Gaussian matrix twists like the identity (PhaseFlow hint); a rank-one
    # outer product does not (RealSmall hint); both hints as the oracle's
    a = np.random.default_rng(4).standard_normal((40, 40))
    (u, s, vt), rep = PhaseEngine.solve_real(a)
    assert rep.passport["route_hint"] == O.triage(a)["passport_route"] == "RealPhaseFlowPolished"
    assert rep.route == "RealSmall" and rep.rel_recon < 4e-13
    r1 = np.outer(np.arange(1.0, 9.0), np.arange(1.0, 9.0))
    (u, s, vt), rep = PhaseEngine.solve_real(r1)
    assert rep.passport["route_hint"] == O.triage(r1)["passport_route"] == "RealSmall"
    assert rep.rel_recon < 4e-13
    rng = np.random.default_rng(2)
    q = np.linalg.qr(rng.standard_normal((10, 10)))[0]
    fam = [q @ np.diag(1.0 + k + np.arange(10) * 0.3) @ q.T for k in range(4)]
    v, diags, trace, rep = PhaseEngine.diagonalize_family(fam)
    assert rep.route == "JointPhaseJade" and rep.passport["family"] == 4 and rep.orth_v < 1e-10
    assert trace.final_offdiag < trace.initial_offdiag * 1e-8


def test_solvers_mirror():  # src/lib.rs:56-60, :117-121
    from lie_cliffalg_analog_svd_b200 import solvers
    a = np.random.default_rng(8).standard_normal((20, 20))
    so = O.LieSvdSmall.solve(a)[1]
    for run in (solvers.run_small, solvers.run_auto):
        u, s, vt, secs = run(a)
        assert secs > 0 and np.max(np.abs(s - so)) <= 1e-13 * so.max()
