"""The multi-rank batched entry on one GPU (no process group): the shard is
the whole batch and the results are the single-call results bit for bit.
Several GPUs are covered on CPU by the gloo ranks of test_dist.py."""
import numpy as np
import pytest

from lie_cliffalg_analog_svd_b200 import profiles as P
from lie_cliffalg_analog_svd_b200 import svd_batched
from lie_cliffalg_analog_svd_b200.dist import svd_batched_sharded

pytestmark = pytest.mark.gpu


def test_sharded_entry_matches_single_call():
    ns, a, _ = P.uneven_batch_workload(3000, seed=9)
    u, s, vt, st, rng = svd_batched_sharded(ns, a)
    u1, s1, vt1, _, st1 = svd_batched(ns, a)
    assert st == st1 and rng == (0, ns.size)
    assert np.array_equal(u, u1) and np.array_equal(s, s1) and np.array_equal(vt, vt1)
