"""The batched kernel's autotuner (lsvd_autotune_f64): it times every
feasible team shape per size class on the device and writes the fastest to
the shape cache; the planner then loads those shapes, and the batched SVD on
them still matches the oracle (FP64 bars of test_gpu_small.py)."""
import numpy as np
import pytest

import oracle as O
from lie_cliffalg_analog_svd_b200 import Context, svd_batched, unpack
from lie_cliffalg_analog_svd_b200 import profiles as P
from lie_cliffalg_analog_svd_b200.api import autotune, class_shapes

pytestmark = pytest.mark.gpu


def test_autotune_writes_cache_and_planner_loads_it(monkeypatch, tmp_path):
    cache = tmp_path / "shapes.json"
    monkeypatch.delenv("LSVD_SHAPES", raising=False)
    monkeypatch.setenv("LSVD_AUTOTUNE_CACHE", str(cache))
    ctx = Context(0)
    default = class_shapes("fp64", ctx=ctx)
    rep = autotune(per_class=96, ctx=ctx)
    assert cache.exists() and '"shapes_fp64": "' in cache.read_text()
    lines = [ln for ln in rep.splitlines() if ln.startswith("class")]
    assert len(lines) == 6, rep
    tuned = class_shapes("fp64", ctx=ctx)
    # the planner reads exactly what the report chose, class by class
    for ln in lines:
        c = int(ln.split()[1])
        chosen = [int(x) for x in ln.split(": ")[1].split()[0].split(",")]
        assert list(tuned[c]) == chosen, (c, tuned[c], chosen)
    assert list(tuned[0]) == list(default[0])  # the micro class is not tuned
    # the batched SVD on the tuned shapes against the oracle
    ns, a, sig = P.uneven_batch_workload(400, seed=71)
    u, s, vt, _, st = svd_batched(ns, a, ctx=ctx)
    assert st == 0
    as_, ss, us, vts = unpack(ns, a), unpack(ns, s, square=False), unpack(ns, u), unpack(ns, vt)
    for t in range(0, len(ns), 7):
        n = int(ns[t])
        so = (O.LieSvdMicro if n <= 4 else O.LieSvdSmall).solve(as_[t])[1]
        assert np.max(np.abs(ss[t] - so)) <= 1e-13 * max(so[0], 1e-300)
        assert np.linalg.norm((us[t] * ss[t]) @ vts[t] - as_[t]) <= 4e-13 * max(np.linalg.norm(as_[t]), 1e-300)
    ctx.close()
