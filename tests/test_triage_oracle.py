"""The oracle's restatement of the reference's triage statistics (the
checker of the GPU triage kernel) against the reference's own tests:
src/lie_svd_phasehealth.rs:351-464, src/lie_svd_adaptive.rs:382-552 and
src/lie_svd_engine.rs:338-358."""
import numpy as np

import oracle as O


def upper_shift(n, d=1.0, u=3.0):
    a = np.zeros((n, n))
    for i in range(n):
        a[i, i] = d
        if i + 1 < n:
            a[i, i + 1] = u
    return a


def test_phase_signature_sees_causal_flow():  # phasehealth :398-403
    t = O.triage(upper_shift(12))
    assert t["causal_disbalance"] > 0.99 and t["max_twist"] > 0.9


def test_phase_signature_accepts_rectangular():  # :405-415
    i, j = np.meshgrid(np.arange(9), np.arange(14), indexing="ij")
    t = O.triage(np.sin((i * 7 + j * 11 + 3).astype(float)))
    assert all(np.isfinite(t[k]) for k in ("mean_stress", "max_twist", "entropy_gap"))
    assert t["route"] is None and t["passport_route"] == "RealSmall"


def test_torsion_energy():  # :417-447
    a = upper_shift(12)
    direct = np.linalg.norm(0.5 * (a - a.T))
    t = O.triage(a)
    assert t["torsion_energy"] > 0 and abs(t["torsion_energy"] - direct) < 1e-9
    i, j = np.meshgrid(np.arange(6), np.arange(6), indexing="ij")
    sym = np.where(i == j, 2.0 + i, 0.1 * (i + j))
    assert O.triage(sym)["torsion_energy"] < 1e-12


def test_phase_entropy_diag_vs_dense():  # :449-464
    diag = np.diag([4.0, 3.0, 2.0, 1.0, 0.5, 0.25])
    i, j = np.meshgrid(np.arange(6), np.arange(6), indexing="ij")
    dense = 1.0 + 0.3 * np.sin((i * 5 + j * 3).astype(float))
    gd, gn = O.triage(diag), O.triage(dense)
    assert gd["phase_entropy"] < gn["phase_entropy"]
    g = O.triage(upper_shift(12))
    assert np.isfinite(g["global_phase"]) and 0 <= g["chirality_balance"] <= 1 and 0 <= g["phase_entropy"] <= 1


def test_engine_passport_global_invariants():  # engine :349-362
    t = O.triage(upper_shift(8))
    assert np.isfinite(t["global_phase"]) and t["torsion_energy"] > 0
    assert 0 <= t["chirality_balance"] <= 1 and 0 <= t["phase_entropy"] <= 1


def _lcg_matrix(n, state=17):
    out = np.empty((n, n))
    mask = (1 << 64) - 1
    for k in range(n * n):
        state = (state * 6364136223846793005 + 1) & mask
        out.flat[k] = 2.0 * ((state >> 11) * (1.0 / (1 << 53))) - 1.0
    return out


def test_adaptive_routes():  # adaptive :395-552
    n = 16
    assert O.triage(np.diag(2.0 - np.arange(n) / n))["route"] == "Small"
    i, j = np.meshgrid(np.arange(24), np.arange(24), indexing="ij")
    stress = np.where(i // 6 == j // 6, 4.0, 0.02) + np.sin(((i + j) * 31).astype(float)) * 1e-3
    assert O.triage(stress)["route"] == "CoreFlowTopo"
    assert O.triage(np.sin((i * 13 + j * 7 + 3).astype(float)))["route"] == "Small"
    assert O.triage(_lcg_matrix(32))["route"] == "Small"
    assert O.triage(upper_shift(24, 1.0, 5.0))["route"] == "PhaseFlow"
    assert O.triage(upper_shift(128, 1.0, 5.0))["route"] == "Small"
    assert O.triage(np.eye(3))["route"] == "Micro"
    assert O.triage(np.random.default_rng(0).standard_normal((600, 600)))["route"] == "Hybrid"
