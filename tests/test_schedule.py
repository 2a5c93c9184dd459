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


# ---- from_real_phaseflow (src/lie_svd_compiler.rs:59-88) and the binary frame

def _reference_phaseflow_cases():
    # the reference's own compiler tests (src/lie_svd_compiler.rs:293-360)
    return [
        ([(2, 0, 1, 0.125, -0.25, "unwrap")], 4),
        ([(0, 2, 3, 0.1, -0.1, "causal_antispin")], 4),
        ([(1, 0, 2, 0.03, 0.0, "cross_phase_yinyang")], 4),
        ([(0, 0, 1, 0.2, 0.1, "phase_conjugate"), (1, 1, 2, -0.05, 0.02, "bottleneck")], 3),
    ]


def _random_phaseflow(rng, count, channels):
    ev = []
    for _ in range(count):
        i, j = sorted(rng.choice(channels, 2, replace=False))
        ev.append((int(rng.integers(0, 40)), int(i), int(j), float(rng.normal()), float(rng.normal()),
                   L.PHASE_ROTOR_KINDS[int(rng.integers(0, 9))]))
    return ev


def test_real_phaseflow_json_identical_to_oracle():
    rng = np.random.default_rng(5)
    cases = _reference_phaseflow_cases() + [(_random_phaseflow(rng, 57, 12), 12), ([], 3)]
    for events, ch in cases:
        for target in ("mzi_mesh", "fpga_rotor_mesh"):
            ours = HardwareSchedule.from_real_phaseflow_json(events, ch, target)
            want = O.HardwareSchedule.from_real_phaseflow(events, ch, target).to_json_string()
            assert ours == want
            js = json.loads(ours)
            assert js["total_events"] == len(events) and "diagonal_signs" not in js
    # the reference tests' own assertions
    js = HardwareSchedule.from_real_phaseflow_json(*_reference_phaseflow_cases()[0])
    assert '"target": "mzi_mesh"' in js and '"kind": "unwrap"' in js
    assert max(e["layer"] for e in json.loads(js)["events"]) + 1 == 3  # conflict_free_layer_count
    for (events, ch), name in zip(_reference_phaseflow_cases()[1:3], ("causal_antispin", "cross_phase_yinyang")):
        assert name in HardwareSchedule.from_real_phaseflow_json(events, ch)


def test_real_phaseflow_rejects_bad_kind():
    with pytest.raises(L.LsvdError):
        HardwareSchedule.from_real_phaseflow_json([(0, 0, 1, 0.1, 0.1, 9)], 2)


def _frame(buf: bytes):
    hdr = np.frombuffer(buf[:64], dtype=L.SCHED_HEADER_DTYPE)[0]
    n = int(hdr["total_events"])
    rec = np.frombuffer(buf[64:64 + 56 * n], dtype=L.SCHED_RECORD_DTYPE)
    signs = np.frombuffer(buf[64 + 56 * n:64 + 56 * n + 8 * int(hdr["n_signs"])], dtype="<f8")
    return hdr, rec, signs


def test_binary_frame_of_phaseflow_round_trips_to_json():
    rng = np.random.default_rng(6)
    for events, ch in _reference_phaseflow_cases() + [(_random_phaseflow(rng, 200, 30), 30), ([], 5)]:
        buf = HardwareSchedule.from_real_phaseflow_binary(events, ch, "fpga_rotor_mesh")
        hdr, rec, signs = _frame(buf)
        assert hdr["magic"] == b"PSCHEDv1" and hdr["header_bytes"] == 64 and hdr["record_bytes"] == 56
        assert hdr["target"] == 1 and hdr["flags"] == 0 and hdr["channels"] == ch
        assert len(buf) == 64 + 56 * len(events) and signs.size == 0
        assert [int(x) for x in rec["layer"]] == [e[0] for e in events]
        assert HardwareSchedule.binary_to_json(buf) == \
            HardwareSchedule.from_real_phaseflow_json(events, ch, "fpga_rotor_mesh")


def _random_stream(rng, channels, rounds):
    rot = []
    for r in range(rounds):
        perm = rng.permutation(channels)
        for k in range(0, channels - 1, 2):
            if rng.random() < 0.7:
                i, j = sorted((int(perm[k]), int(perm[k + 1])))
                rot.append((i, j, r, float(rng.normal())))
    out = np.zeros(len(rot), dtype=L.ROTOR_DTYPE)
    out[:] = rot
    return out


def test_binary_frame_of_rotor_stream_matches_json_entry():
    rng = np.random.default_rng(7)
    for channels, rounds in ((2, 1), (6, 3), (17, 9), (64, 40)):
        rot = _random_stream(rng, channels, rounds)
        buf = HardwareSchedule.from_rotor_stream_binary(rot, channels)
        hdr, rec, signs = _frame(buf)
        assert hdr["flags"] == L.SCHED_CANONICAL and hdr["n_signs"] == channels and np.all(signs == 1.0)
        # stream order kept in the frame, (round, i, j) order in the JSON
        assert np.array_equal(rec["layer"], rot["round"]) and np.array_equal(rec["i"], rot["j"])
        assert np.array_equal(rec["theta"], -rot["theta"])
        assert HardwareSchedule.binary_to_json(buf) == HardwareSchedule.from_rotor_stream_json(rot, channels)


def test_binary_frame_energy_section_and_malformed_frames():
    events = [(0, 0, 1, 0.3, 0.1, "surgery"), (1, 1, 2, -0.2, 0.4, "directional")]
    buf = bytearray(HardwareSchedule.from_real_phaseflow_binary(events, 3))
    # add the optional energy section: event 0 has both, event 1 only energy_after
    hdr = np.frombuffer(bytes(buf[:64]), dtype=L.SCHED_HEADER_DTYPE).copy()
    hdr["flags"] = L.SCHED_ENERGY
    energy = np.array([1.5, 0.25, np.nan, 2.0], dtype="<f8")
    full = hdr.tobytes() + bytes(buf[64:]) + energy.tobytes()
    js = json.loads(HardwareSchedule.binary_to_json(full))
    assert js["events"][0]["energy_before"] == 1.5 and js["events"][0]["energy_after"] == 0.25
    assert "energy_before" not in js["events"][1] and js["events"][1]["energy_after"] == 2.0
    ref = O.HardwareSchedule.from_real_phaseflow(events, 3)
    ref.events[0].energy_before, ref.events[0].energy_after, ref.events[1].energy_after = 1.5, 0.25, 2.0
    assert HardwareSchedule.binary_to_json(full) == ref.to_json_string()
    for bad in (bytes(buf[:-1]), b"XSCHEDv1" + bytes(buf[8:]), bytes(buf[:60])):
        with pytest.raises(L.LsvdError):
            HardwareSchedule.binary_to_json(bad)
    bad_kind = bytearray(buf)
    bad_kind[64 + 49] = 200  # kind code of record 0
    with pytest.raises(L.LsvdError):
        HardwareSchedule.binary_to_json(bytes(bad_kind))
