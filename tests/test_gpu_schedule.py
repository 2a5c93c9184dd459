"""The binary phase-schedule frame written on the device from a rotor stream
in HBM (lsvd_schedule_binary_from_rotors with LSVD_DEVICE_POINTERS) against
the host encoder of the same stream: byte-identical frames, and the frame's
JSON equal to the rotor-stream JSON entry (src/lie_svd_compiler.rs:213-265)."""
import numpy as np
import pytest

from lie_cliffalg_analog_svd_b200 import HardwareSchedule, LieSvdSmall
from lie_cliffalg_analog_svd_b200 import _lib as L
from lie_cliffalg_analog_svd_b200 import profiles as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _device(rot):
    return torch.from_numpy(rot.view(np.uint8).copy()).cuda()


def test_device_frame_of_solver_stream_matches_host():
    a = P.generate(64, "uniform_random", 11)[0]
    r = LieSvdSmall.solve_full(a, rotor_cap=1 << 17)
    rot = r.rotors
    assert rot.size > 1000
    host = HardwareSchedule.from_rotor_stream_binary(rot, 64)
    dev = HardwareSchedule.from_rotor_stream_binary(_device(rot), 64)
    assert dev.is_cuda and bytes(dev.cpu().numpy()) == host
    assert HardwareSchedule.binary_to_json(dev) == HardwareSchedule.from_rotor_stream_json(rot, 64)


@pytest.mark.parametrize("count,channels", [(0, 64), (1, 2), (255, 512), (256, 64), (300_001, 1000)])
def test_device_frame_sizes(count, channels):
    rng = np.random.default_rng(count)
    rot = np.zeros(count, dtype=L.ROTOR_DTYPE)
    if count:
        i = rng.integers(0, channels - 1, count)
        j = i + 1 + (rng.integers(0, 1 << 30, count) % (channels - 1 - i))
        rot["i"], rot["j"] = i, j
        rot["round"] = np.sort(rng.integers(0, 1 << 20, count))
        rot["theta"] = rng.normal(size=count)
    host = HardwareSchedule.from_rotor_stream_binary(rot, channels)
    dev = HardwareSchedule.from_rotor_stream_binary(_device(rot) if count else
                                                    torch.zeros(0, dtype=torch.uint8, device="cuda"), channels)
    assert bytes(dev.cpu().numpy()) == host


def test_device_frame_rejects_bad_rotor():
    rot = np.zeros(3, dtype=L.ROTOR_DTYPE)
    rot[:] = [(0, 1, 0, 0.1), (5, 2, 0, 0.2), (1, 3, 1, 0.3)]  # i >= j in the second
    with pytest.raises(L.LsvdError):
        HardwareSchedule.from_rotor_stream_binary(_device(rot), 8)
