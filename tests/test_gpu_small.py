"""GPU parity: the CUDA small/micro/batched SVD against the oracle (CPU
restatement of src/lie_svd_small.rs / src/lie_svd_micro.rs) on identical
seeded inputs, plus the reference's own hot-path tests run on the GPU.

Tolerances (FP64 path):
* singular values, normwise:  max|s_gpu - s_ref| / s_ref[0] <= 1e-13
* orthogonality ||U^T U - I||_F, ||V^T V - I||_F and relative reconstruction
  <= max(1e-13, 8 x the oracle's own value on the same input)
* singular vectors: |<u_gpu_j, u_ref_j>| >= 1 - 1e-9 for columns whose
  singular value is separated from its neighbours by a relative gap > 1e-6
"""
import numpy as np
import pytest

import oracle as O
from lie_cliffalg_analog_svd_b200 import LieSvd, LieSvdMicro, LieSvdSmall, metrics, svd_batched, unpack
from lie_cliffalg_analog_svd_b200 import _lib as L
from lie_cliffalg_analog_svd_b200 import profiles as P

pytestmark = pytest.mark.gpu


def mets(a, u, s, vt):
    rec = np.linalg.norm((u * s) @ vt - a) / max(np.linalg.norm(a), 1e-300)
    return rec, np.linalg.norm(u.T @ u - np.eye(u.shape[1])), np.linalg.norm(vt @ vt.T - np.eye(vt.shape[0]))


def sigma_err(s, ref):
    s, ref = np.sort(s)[::-1], np.sort(ref)[::-1]
    return np.max(np.abs(s - ref)) / max(ref[0], 1e-300)


def check_vs_oracle(a, tol_sigma=1e-13, vec_tol=1e-9):
    ug, sg, vg = LieSvdSmall.solve(a)
    uo, so, vo = O.LieSvdSmall.solve(a)
    assert np.all(np.isfinite(ug)) and np.all(np.isfinite(vg)) and np.all(sg >= 0)
    assert np.all(np.diff(sg) <= 0), "sigma must be descending"
    assert sigma_err(sg, so) <= tol_sigma
    rg, oug, ovg = mets(a, ug, sg, vg)
    ro, ouo, ovo = mets(a, uo, so, vo)
    # both solvers stop at off(P) < 1e-13 ||P||_F (src/lie_svd_small.rs:226): the residual
    # left by the last sweep lands anywhere below that, so the bar is absolute
    assert rg <= max(4e-13, 8 * ro), (rg, ro)
    assert oug <= max(1e-13, 8 * ouo), (oug, ouo)
    assert ovg <= max(1e-13, 8 * ovo), (ovg, ovo)
    n = a.shape[0]
    s = so
    for j in range(n):
        gap = min([abs(s[j] - s[k]) for k in (j - 1, j + 1) if 0 <= k < n] + [np.inf])
        if s[j] > 1e-6 * s[0] and gap > 1e-6 * s[0]:
            assert abs(ug[:, j] @ uo[:, j]) >= 1 - vec_tol, j
            assert abs(vg[j] @ vo[j]) >= 1 - vec_tol, j
    return ug, sg, vg


@pytest.mark.parametrize("n", list(range(1, 65)))
def test_random_gaussian_every_size(n):
    a = np.random.default_rng(1000 + n).standard_normal((n, n))
    check_vs_oracle(a)


def test_config1_64_gaussian_with_rotor_stream():
    a = np.random.default_rng(17).standard_normal((64, 64))
    check_vs_oracle(a)
    r = LieSvdSmall.solve_full(a, rotor_cap=200_000)
    assert r.diag["rotor_count"] == r.diag["rotations"] > 0
    # rebuild V from the stream: V = prod of column rotations, then permute
    rot = np.sort(r.rotors, order=["round", "i", "j"])
    v = np.eye(64)
    for e in rot:
        i, j, th = int(e["i"]), int(e["j"]), float(e["theta"])
        c, s = np.cos(th), np.sin(th)
        vi, vj = v[:, i].copy(), v[:, j].copy()
        v[:, i] = c * vi - s * vj
        v[:, j] = s * vi + c * vj
    v = v[:, r.perm]
    assert np.max(np.abs(v - r.vt.T)) < 1e-11
    # layers are conflict-free: no channel twice in one round
    for rd in np.unique(rot["round"]):
        ch = np.concatenate([rot[rot["round"] == rd]["i"], rot[rot["round"] == rd]["j"]])
        assert ch.size == np.unique(ch).size
    assert r.diag["orth_u"] < 1e-13 and r.diag["orth_v"] < 1e-13 and r.diag["rel_recon"] < 5e-14


# --- the reference's own tests (src/lie_svd_small.rs:543-657) on the GPU ----

def test_ref_random_64():
    a = np.random.default_rng(7).uniform(-1, 1, (64, 64))
    u, s, vt = check_vs_oracle(a)
    r, ou, ov = mets(a, u, s, vt)
    assert r < 1e-8 and ou < 1e-8 and ov < 1e-8


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 9, 13, 17, 31])
def test_ref_odd_sizes(n):
    check_vs_oracle(np.random.default_rng(100 + n).uniform(-1, 1, (n, n)))


def test_ref_ill_conditioned_32():
    n = 32
    rng = np.random.default_rng(42)
    u0, v0 = P.random_orthogonal(n, rng), P.random_orthogonal(n, rng)
    a = (u0 * 10.0 ** (-15.0 * np.arange(n) / (n - 1))) @ v0.T
    u, s, vt = LieSvdSmall.solve(a)
    r, ou, ov = mets(a, u, s, vt)
    assert r < 1e-6 and ou < 1e-6 and ov < 1e-6
    assert sigma_err(s, O.LieSvdSmall.solve(a)[1]) < 1e-13


def test_ref_jordan_64():
    a, _ = P.generate(64, "jordan_defective", 0)
    check_vs_oracle(a)


@pytest.mark.parametrize("n", [16, 64])
def test_ref_pei_closed_form(n):
    a = P.pei_matrix(n, 0.01)
    u, s, vt = LieSvdSmall.solve(a)
    m = metrics.compute(a, u, s, vt, P.pei_matrix_singular_values(n, 0.01))
    assert m.orth_u < 1e-9 and m.orth_v < 1e-9 and m.rel_recon < 1e-9
    assert m.sigma_max_rel < 1e-8 and m.sigma_tail_rel < 1e-6


@pytest.mark.parametrize("profile", P.PROFILES)
@pytest.mark.parametrize("n", [32, 64])
def test_profiles(profile, n):
    a, ref = P.generate(n, profile, 909)
    u, s, vt = LieSvdSmall.solve(a)
    m = metrics.compute(a, u, s, vt, ref)
    assert m.orth_u < 1e-9 and m.orth_v < 1e-9 and m.rel_recon < 1e-9
    so = O.LieSvdSmall.solve(a)[1]
    assert sigma_err(s, so) < 1e-13
    if profile == "extreme_ill_conditioned":
        assert np.all(np.abs(np.sort(s)[::-1] - ref) < 1e-9)


def test_named_matrices():
    import json, os
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "named_sigma.json")))
    build = {"kahan": lambda n, p: P.kahan_matrix(n, float(p)), "hilbert": lambda n, p: P.hilbert_matrix(n),
             "pei": lambda n, p: P.pei_matrix(n, float(p)), "frank": lambda n, p: P.frank_matrix(n),
             "parter": lambda n, p: P.parter_matrix(n), "cauchy": lambda n, p: P.cauchy_matrix(n),
             "vandermonde": lambda n, p: P.vandermonde_matrix(n)}
    for name, rec in gold.items():
        parts = name.split("_")
        a = build[parts[0]](rec["n"], parts[2] if len(parts) > 2 else None)
        want = np.array([float(x) for x in rec["sigma"]])
        u, s, vt = LieSvdSmall.solve(a)
        assert sigma_err(s, want) < 1e-13, name
        r, ou, ov = mets(a, u, s, vt)
        assert r < 1e-9 and ou < 1e-9 and ov < 1e-9, name


# --- edge cases ---------------------------------------------------------------

def test_zero_matrix_gives_orthogonal_bases():
    for n in (1, 5, 64):
        a = np.zeros((n, n))
        u, s, vt = LieSvdSmall.solve(a)
        assert np.all(s == 0)
        assert np.linalg.norm(u.T @ u - np.eye(n)) < 1e-12
        assert np.linalg.norm(vt @ vt.T - np.eye(n)) < 1e-12


def test_nonfinite_input_reports_status():
    a = np.random.default_rng(0).standard_normal((8, 8))
    a[3, 4] = np.nan
    r = LieSvdSmall.solve_full(a)
    assert r.diag["status"] == L.NONFINITE_INPUT
    assert r.diag["flags"] & L.MAT_NONFINITE
    assert np.all(np.isnan(r.sigma))


def test_rank_deficient_and_repeated():
    rng = np.random.default_rng(5)
    n = 40
    x = rng.standard_normal((n, 3))
    check_vs_oracle(x @ rng.standard_normal((3, n)), tol_sigma=1e-13)
    u0, v0 = P.random_orthogonal(n, rng), P.random_orthogonal(n, rng)
    s0 = np.repeat([3.0, 2.0, 1.0, 0.5], 10)
    a = (u0 * s0) @ v0.T
    u, s, vt = LieSvdSmall.solve(a)
    assert sigma_err(s, s0) < 1e-13
    r, ou, ov = mets(a, u, s, vt)
    ro, ouo, ovo = mets(a, *O.LieSvdSmall.solve(a))
    assert r < max(4e-13, 8 * ro) and ou < max(2e-13, 8 * ouo) and ov < max(2e-13, 8 * ovo)


def test_subnormal_and_dynamic_range():
    i, j = np.meshgrid(np.arange(6), np.arange(6), indexing="ij")
    a = 1e-310 * np.sin((i * 3 + j + 1).astype(float))
    u, s, vt = LieSvdSmall.solve(a)
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(vt)) and np.all((s == 0) | (s < 1e-300))
    assert np.linalg.norm(u.T @ u - np.eye(6)) < 1e-9
    rng = np.random.default_rng(99)
    n = 16
    u0, v0 = P.random_orthogonal(n, rng), P.random_orthogonal(n, rng)
    a = (u0 * 10.0 ** (150.0 * (1 - 2 * np.arange(n) / (n - 1)))) @ v0.T
    u, s, vt = LieSvdSmall.solve(a)
    m = metrics.compute(a, u, s, vt)
    assert m.orth_u < 1e-9 and m.orth_v < 1e-9 and m.rel_recon < 1e-9


def test_bad_shapes_raise():
    with pytest.raises(L.LsvdError):
        LieSvdSmall.solve(np.zeros((3, 4)))
    with pytest.raises(L.LsvdError):
        LieSvdMicro.solve(np.zeros((5, 5)))


def test_deterministic_replay():
    a = np.random.default_rng(3).standard_normal((50, 50))
    r1 = LieSvdSmall.solve(a)
    r2 = LieSvdSmall.solve(a)
    for x, y in zip(r1, r2):
        assert np.array_equal(x, y)


# --- micro (src/lie_svd_micro.rs:238-267) ------------------------------------

@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_micro_matches_oracle(n):
    rng = np.random.default_rng(900 + n)
    for _ in range(32):
        a = rng.uniform(-2, 2, (n, n))
        ug, sg, vg = LieSvdMicro.solve(a)
        uo, so, vo = O.LieSvdMicro.solve(a)
        # same fixed schedule and sign convention as the reference
        assert np.max(np.abs(sg - so)) <= 1e-14 * max(so[0], 1)
        assert np.max(np.abs(ug - uo)) < 1e-12 and np.max(np.abs(vg - vo)) < 1e-12
        r, ou, ov = mets(a, ug, sg, vg)
        assert r < 1e-10 and ou < 1e-10 and ov < 1e-10


def test_micro_degenerate_4():
    a = np.zeros((4, 4))
    a[0, 0] = a[1, 1] = 10.0
    a[2, 2] = a[3, 3] = 1e-12
    a[0, 1] = 0.25
    a[2, 3] = -0.5
    u, s, vt = LieSvdMicro.solve(a)
    r, ou, ov = mets(a, u, s, vt)
    assert r < 1e-10 and ou < 1e-10 and ov < 1e-10


def test_dispatcher_routes():
    for n in (2, 4, 5, 20):
        a = np.random.default_rng(n).standard_normal((n, n))
        u, s, vt = LieSvd.solve(a)
        assert sigma_err(s, np.linalg.svd(a, compute_uv=False)) < 1e-13


# --- rectangular (src/lie_svd_small.rs:462-540) -------------------------------

def test_rectangular_cases():
    rng = np.random.default_rng(2026)
    cases = [rng.uniform(-1, 1, (30, 3)), rng.uniform(-1, 1, (20, 15)),
             np.cos((np.arange(4)[:, None] * 5 + np.arange(11)[None, :] * 3 + 2).astype(float)),
             rng.standard_normal((128, 64)), rng.standard_normal((64, 100))]
    for a in cases:
        u, s, vt = LieSvdSmall.solve_rectangular(a)
        uo, so, vo = O.LieSvdSmall.solve_rectangular(a)
        k = min(a.shape)
        assert u.shape == (a.shape[0], k) and vt.shape == (k, a.shape[1])
        assert np.linalg.norm((u * s) @ vt - a) / np.linalg.norm(a) < 1e-12
        assert np.linalg.norm(u.T @ u - np.eye(k)) < 1e-12
        assert sigma_err(s, so) < 1e-13


def test_rectangular_rank_deficient_column():
    n = 20
    i = np.arange(n)
    v = np.sin((i * 11 + 3) * 0.23) * 2.0
    a = np.stack([v, np.cos((i * 13 + 7) * 0.41), v], axis=1)
    u, s, vt = LieSvdSmall.solve_rectangular(a)
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(s)) and np.all(np.isfinite(vt))
    assert np.linalg.norm((u * s) @ vt - a) / np.linalg.norm(a) < 1e-8


# --- batched ------------------------------------------------------------------

def test_batched_matches_single_and_oracle():
    ns, a, sig = P.uneven_batch_workload(3000, seed=5)
    u, s, vt, dg, st = svd_batched(ns, a, want_diag=True)
    assert st == L.OK
    us, ss, vts = unpack(ns, u), unpack(ns, s, square=False), unpack(ns, vt)
    as_ = unpack(ns, a)
    sr = unpack(ns, sig, square=False)
    rng = np.random.default_rng(0)
    for t in rng.choice(len(ns), 120, replace=False):
        n = int(ns[t])
        assert dg[t]["route"] == (L.ROUTE_MICRO if n <= 4 else L.ROUTE_SMALL)
        uo, so, vo = O.LieSvdMicro.solve(as_[t]) if n <= 4 else O.LieSvdSmall.solve(as_[t])
        assert sigma_err(ss[t], so) < 1e-13, (t, n)
        assert sigma_err(ss[t], sr[t]) < 1e-13, (t, n)
        r, ou, ov = mets(as_[t], us[t], ss[t], vts[t])
        ro, ouo, ovo = mets(as_[t], uo, so, vo)
        assert r < max(4e-13, 8 * ro) and ou < 2e-13 and ov < 2e-13, (t, n, r, ro, ou, ov)
        assert abs(dg[t]["orth_u"] - ou) < 1e-14 + 1e-3 * ou
    assert np.all(dg["orth_u"] < 2e-13) and np.all(dg["orth_v"] < 2e-13)
    assert np.all(dg["rel_recon"] < 4e-13)


def test_batched_device_pointers_and_determinism():
    import torch
    ns, a, _ = P.uneven_batch_workload(500, seed=9)
    ah = svd_batched(ns, a)
    ad = torch.from_numpy(a).cuda()
    u, s, vt, _, st = svd_batched(ns, ad)
    torch.cuda.synchronize()
    assert st == L.OK
    assert np.array_equal(u.cpu().numpy(), ah[0]) and np.array_equal(s.cpu().numpy(), ah[1])
    u2, s2, vt2, _, _ = svd_batched(ns, ad)
    assert torch.equal(u, u2) and torch.equal(vt, vt2)


def test_batched_edge_cases():
    ns = np.array([1, 1, 2, 3, 4, 5, 64, 33, 1], dtype=np.int32)
    rng = np.random.default_rng(1)
    mats = [rng.standard_normal((n, n)) for n in ns]
    mats[1][:] = 0.0
    mats[5][:] = 0.0
    a = np.concatenate([m.ravel() for m in mats])
    u, s, vt, dg, st = svd_batched(ns, a, want_diag=True)
    assert st == L.OK
    for t, (m, ut, st_, vtt) in enumerate(zip(mats, unpack(ns, u), unpack(ns, s, False), unpack(ns, vt))):
        ref = np.linalg.svd(m, compute_uv=False)
        assert sigma_err(st_, ref) < 1e-13 if ref[0] > 0 else np.all(st_ == 0)
        assert np.linalg.norm(ut.T @ ut - np.eye(len(st_))) < 1e-12
    bad = a.copy()
    bad[0] = np.inf
    *_, st = svd_batched(ns, bad)
    assert st == L.NONFINITE_INPUT
    with pytest.raises(L.LsvdError):
        svd_batched(np.array([65], dtype=np.int32), np.zeros(65 * 65))


def test_metrics_match_oracle():
    rng = np.random.default_rng(8)
    a = rng.standard_normal((30, 30))
    u, s, vt = O.LieSvdSmall.solve(a)
    ref = np.linalg.svd(a, compute_uv=False)
    mg = metrics.compute(a, u, s, vt, ref)
    mo = O.metrics.compute(a, u, s, vt, ref)
    for f in ("rel_recon", "orth_u", "orth_v", "sigma_max_rel", "sigma_tail_rel"):
        x, y = getattr(mg, f), getattr(mo, f)
        assert abs(x - y) <= 1e-3 * abs(y) + 1e-18, f


def test_batched_host_pipeline_matches_device():
    # >= 16384 matrices from host memory take the chunked, copy-overlapped
    # path; every matrix is solved independently, so the results must equal
    # the device-pointer (single plan) call bit for bit
    import torch
    ns, a, sig = P.uneven_batch_workload(20000, seed=77, n_lo=2, n_hi=24)
    pin = lambda k: torch.empty(k, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    a_h = pin(a.size)
    a_h[:] = a
    so = int(ns.astype(np.int64).sum())
    out_h = (pin(a.size), pin(so), pin(a.size), np.empty(ns.size, dtype=L.DIAG_DTYPE))
    u, s, vt, dg, st = svd_batched(ns, a_h, want_diag=True, out=out_h)
    assert st == 0
    ud, sd, vtd, dgd, std = svd_batched(ns, torch.from_numpy(a).cuda(), want_diag=True)
    assert std == 0
    assert np.array_equal(s, sd.cpu().numpy())
    assert np.array_equal(u, ud.cpu().numpy()) and np.array_equal(vt, vtd.cpu().numpy())
    dgd = np.frombuffer(dgd.cpu().numpy().tobytes(), dtype=L.DIAG_DTYPE)
    assert np.array_equal(dg["rotations"], dgd["rotations"])
    first = np.concatenate([[0], np.cumsum(ns)[:-1]])
    assert np.max(np.abs(s - sig) / np.repeat(sig[first], ns)) <= 1e-13
    # pageable host memory takes the same path (its copies are then synchronous)
    u2, s2, vt2, _, st2 = svd_batched(ns, a)
    assert st2 == 0 and np.array_equal(s2, s)


def test_batched_host_pipeline_uniform_n_matches_device():
    # a uniform size list gives chunks with equal size lists: each chunk must
    # still stage through its own buffers (results bit-identical to the
    # device-pointer call)
    import torch
    count, n = 16384, 16
    ns = np.full(count, n, dtype=np.int32)
    a = np.random.default_rng(123).standard_normal(count * n * n)
    pin = lambda k: torch.empty(k, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    a_h = pin(a.size)
    a_h[:] = a
    out_h = (pin(a.size), pin(count * n), pin(a.size), None)
    u, s, vt, _, st = svd_batched(ns, a_h, out=out_h)
    assert st == 0
    ud, sd, vtd, _, std = svd_batched(ns, torch.from_numpy(a).cuda())
    assert std == 0
    assert np.array_equal(s, sd.cpu().numpy())
    assert np.array_equal(u, ud.cpu().numpy()) and np.array_equal(vt, vtd.cpu().numpy())
    # a second call reuses the per-chunk plans and must give the same bits
    u2, s2, vt2, _, st2 = svd_batched(ns, a_h, out=(pin(a.size), pin(count * n), pin(a.size), None))
    assert st2 == 0 and np.array_equal(s2, s) and np.array_equal(u2, u)


def test_batched_timed_mode_matches_oracle():
    # the benchmark's mode (no LSVD_WANT_DIAG): U, S and Vt of >= 1000
    # matrices across n = 2..64 with the kappa <= 1e12 / degenerate mix,
    # checked against the oracle matrix by matrix
    import concurrent.futures as cf
    ns, a, sig = P.uneven_batch_workload(1200, seed=2024)
    u, s, vt, _, st = svd_batched(ns, a)
    assert st == L.OK
    us, ss, vts, as_ = unpack(ns, u), unpack(ns, s, square=False), unpack(ns, vt), unpack(ns, a)

    def one(t):
        n = int(ns[t])
        uo, so, vo = O.LieSvdMicro.solve(as_[t]) if n <= 4 else O.LieSvdSmall.solve(as_[t])
        return t, uo, so, vo

    with cf.ThreadPoolExecutor(8) as ex:
        res = list(ex.map(one, range(len(ns))))
    for t, uo, so, vo in res:
        n = int(ns[t])
        assert sigma_err(ss[t], so) < 1e-13, (t, n)
        r, ou, ov = mets(as_[t], us[t], ss[t], vts[t])
        ro, ouo, ovo = mets(as_[t], uo, so, vo)
        assert r < max(4e-13, 8 * ro) and ou < max(2e-13, 8 * ouo) and ov < max(2e-13, 8 * ovo), (t, n)
        # separated singular directions agree with the oracle's up to sign
        for j in range(n):
            gap = min([abs(so[j] - so[k]) for k in (j - 1, j + 1) if 0 <= k < n] + [np.inf])
            if so[j] > 1e-6 * so[0] and gap > 1e-6 * so[0]:
                assert abs(us[t][:, j] @ uo[:, j]) >= 1 - 1e-9, (t, n, j)
                assert abs(vts[t][j] @ vo[j]) >= 1 - 1e-9, (t, n, j)
