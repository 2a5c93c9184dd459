"""lsvd_svd_batched_noalloc_f64: the batched FP64 SVD for callers that cannot
allocate device memory (latency-critical loops that cannot take the
device-wide synchronisation of cudaMalloc/cudaFree; hosts whose device memory
belongs to their own allocator).  The entry point keeps its working memory in
a static device array; this test hands it preallocated device buffers through
the C ABI and checks its output against lsvd_svd_batched_f64 on two calls in
a row (the static array keeps the previous call's contents, so the second
call checks that everything is rebuilt and cleared).

Tolerance: the FP64 path's own bars -- singular values within 1e-13
normwise, U/V/reconstruction within 1e-12 -- since both entry points run the
same kernels on the same schedule classes.

This file is collected last (tests/test_zz_*) so that a failure here leaves
every other test already run."""
import ctypes as C

import numpy as np
import pytest

from lie_cliffalg_analog_svd_b200 import _lib as L
from lie_cliffalg_analog_svd_b200 import profiles as P
from lie_cliffalg_analog_svd_b200 import svd_batched

pytestmark = pytest.mark.gpu


def _noalloc(lib, stream, ns, a_dev, u, s, vt, dg):
    nsa = np.ascontiguousarray(ns, dtype=np.int32)
    return lib.lsvd_svd_batched_noalloc_f64(
        C.c_void_p(stream), nsa.size, C.c_void_p(nsa.ctypes.data), C.c_void_p(a_dev.data_ptr()),
        C.c_void_p(u.data_ptr()), C.c_void_p(s.data_ptr()), C.c_void_p(vt.data_ptr()),
        C.c_void_p(dg.data_ptr()), L.WANT_DIAG)


def test_noalloc_matches_batched_twice(monkeypatch, tmp_path):
    import torch
    from lie_cliffalg_analog_svd_b200 import Context
    # both entry points on the built-in team shapes: no LSVD_SHAPES override,
    # no autotune cache, a fresh context (no plan cached under other shapes)
    monkeypatch.delenv("LSVD_SHAPES", raising=False)
    monkeypatch.setenv("LSVD_AUTOTUNE_CACHE", str(tmp_path / "none.json"))
    ctx = Context(0)
    lib = L.load()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for seed, count in ((31, 3000), (32, 1200)):
        ns, a, _ = P.uneven_batch_workload(count, seed=seed)
        ref_u, ref_s, ref_vt, ref_dg, st = svd_batched(ns, a, want_diag=True, ctx=ctx)
        assert st == L.OK
        ad = torch.from_numpy(a).to(dev)
        u = torch.empty_like(ad)
        vt = torch.empty_like(ad)
        s = torch.empty(int(ns.astype(np.int64).sum()), dtype=torch.float64, device=dev)
        dg = torch.empty(count * C.sizeof(L.Diag), dtype=torch.uint8, device=dev)
        assert _noalloc(lib, stream, ns, ad, u, s, vt, dg) == L.OK
        torch.cuda.synchronize()
        s_h = s.cpu().numpy()
        assert np.max(np.abs(s_h - ref_s)) <= 1e-13 * max(1.0, float(np.max(np.abs(ref_s))))
        assert np.max(np.abs(u.cpu().numpy() - ref_u)) < 1e-12
        assert np.max(np.abs(vt.cpu().numpy() - ref_vt)) < 1e-12
        d = np.frombuffer(dg.cpu().numpy().tobytes(), dtype=L.DIAG_DTYPE)
        assert np.all(d["orth_u"] < 4e-13) and np.all(d["rel_recon"] < 4e-13)
        assert np.array_equal(d["route"], ref_dg["route"])
    ctx.close()


def test_noalloc_rejects_too_many_matrices():
    import torch
    lib = L.load()
    count = L_MAX = 65536 + 1
    ns = np.full(count, 2, dtype=np.int32)
    z = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = lib.lsvd_svd_batched_noalloc_f64(None, count, C.c_void_p(ns.ctypes.data),
                                          C.c_void_p(z.data_ptr()), C.c_void_p(z.data_ptr()),
                                          C.c_void_p(z.data_ptr()), C.c_void_p(z.data_ptr()), None, 0)
    assert st == L.UNSUPPORTED and L_MAX == count
