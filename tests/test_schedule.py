"""phase-schedule-v1 compiler (src/lie_svd_compiler.rs) in the library vs
the oracle restatement: byte-identical JSON for identical input matrices,
and the reference's reconstruction rule (src/lie_svd_compiler.rs:396-411)
applied to the library's rotor-stream schedule.  Host-side; no GPU."""
import json
import math

import numpy as np
import pytest

import oracle as O
from lie_cliffalg_analog_svd_b200 import HardwareSchedule
from lie_cliffalg_analog_svd_b200 import _lib as L
from lie_cliffalg_analog_svd_b200 import build as B
from lie_cliffalg_analog_svd_b200 import profiles as P


@pytest.fixture(scope="module", autouse=True)
def _built():
    B.build()


def reconstruct(events, signs):
    d = len(signs)
    rec = np.diag(np.asarray(signs, dtype=float))
    for e in reversed(events):
        c, s = math.cos(e["theta_l"]), math.sin(e["theta_l"])
        i, j = e["i"], e["j"]
        rj, ri = rec[j].copy(), rec[i].copy()
        rec[j] = c * rj - s * ri
        rec[i] = s * rj + c * ri
    return rec


@pytest.mark.parametrize("d", [1, 2, 3, 5, 8, 13])
def test_from_orthogonal_json_identical_to_oracle(d):
    rng = np.random.default_rng(300 + d)
    for v in (P.random_orthogonal(d, rng), np.eye(d), -np.eye(d)[::-1].copy()):
        ours = HardwareSchedule.from_orthogonal_matrix_json(v)
        want = O.HardwareSchedule.from_orthogonal_matrix(v).to_json_string()
        assert ours == want
        js = json.loads(ours)
        assert js["format_version"] == "phase-schedule-v1" and js["channels"] == d
        assert np.max(np.abs(reconstruct(js["events"], js["diagonal_signs"]) - v)) < 1e-12


def test_fpga_target_and_sizing():
    v = P.random_orthogonal(4, np.random.default_rng(1))
    js = HardwareSchedule.from_orthogonal_matrix_json(v, target="fpga_rotor_mesh")
    assert '"target": "fpga_rotor_mesh"' in js


def test_rotor_stream_schedule_reconstructs():
    # a synthetic conflict-free stream: two rounds of rotations on 6 channels
    rot = np.zeros(5, dtype=L.ROTOR_DTYPE)
    rot[:] = [(0, 1, 0, 0.3), (2, 3, 0, -0.7), (4, 5, 0, 1.1), (1, 2, 1, 0.25), (0, 5, 1, -0.4)]
    v = np.eye(6)
    for e in rot:  # the lsvd_rotor convention: V <- V G(i, j, theta)
        i, j, th = int(e["i"]), int(e["j"]), float(e["theta"])
        c, s = math.cos(th), math.sin(th)
        vi, vj = v[:, i].copy(), v[:, j].copy()
        v[:, i] = c * vi - s * vj
        v[:, j] = s * vi + c * vj
    js = json.loads(HardwareSchedule.from_rotor_stream_json(rot, 6))
    assert js["total_events"] == 5
    assert max(e["layer"] for e in js["events"]) + 1 == 2
    assert all(e["source"] == "gpu_jacobi" for e in js["events"])
    assert np.max(np.abs(reconstruct(js["events"], js["diagonal_signs"]) - v)) < 1e-14


def test_rotor_stream_rejects_bad_channels():
    rot = np.zeros(1, dtype=L.ROTOR_DTYPE)
    rot[:] = [(3, 2, 0, 0.1)]
    with pytest.raises(L.LsvdError):
        HardwareSchedule.from_rotor_stream_json(rot, 4)
