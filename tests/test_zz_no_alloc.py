"""GPU: falcon_search_noalloc, the search for callers that cannot allocate
device memory on their query path (fixed-budget serving threads, hosts whose
own runtime owns every device allocation, loops that cannot take the implicit
synchronisation of cudaMalloc/cudaFree).  It keeps its scratch in one static
4 MiB device array instead of cudaMallocAsync.

Its results must equal falcon_search's (the existing entry point) bit for
bit, on two calls in a row, since the static scratch keeps the previous
call's contents.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from helpers import small_graph

pytestmark = pytest.mark.gpu


def _reference(lib, ix, q, params, per_query, k_stride):
    """falcon_search, the existing entry point, on host buffers."""
    from falcon_b200 import _lib
    nq = q.shape[0]
    ids = np.full((nq, k_stride), -7, dtype=np.int32)
    dists = np.zeros((nq, k_stride), dtype=np.float32)
    hops = np.zeros(nq, dtype=np.int32)
    vis = np.zeros(nq, dtype=np.int32)
    pptr = ctypes.cast(params, ctypes.POINTER(_lib.SearchParams)) if per_query else ctypes.byref(params)
    rc = lib.falcon_search(ix._h, q.ctypes.data, nq, q.shape[1], None, pptr, 1 if per_query else 0, ids.ctypes.data,
                           dists.ctypes.data, k_stride, hops.ctypes.data, vis.ctypes.data, _lib.MEM_HOST, None)
    return rc, ids, dists, hops, vis


def _run(lib, fn, ix, dq, params, per_query, k_stride):
    import torch
    from falcon_b200 import _lib
    nq = dq.shape[0]
    ids = torch.full((nq, k_stride), -7, dtype=torch.int32, device=dq.device)
    dists = torch.zeros((nq, k_stride), dtype=torch.float32, device=dq.device)
    hops = torch.zeros(nq, dtype=torch.int32, device=dq.device)
    vis = torch.zeros(nq, dtype=torch.int32, device=dq.device)
    s = torch.cuda.current_stream().cuda_stream
    pptr = ctypes.cast(params, ctypes.POINTER(_lib.SearchParams)) if per_query else ctypes.byref(params)
    args = [ix._h, dq.data_ptr(), nq, dq.stride(0), None, pptr, 1 if per_query else 0, ids.data_ptr(),
            dists.data_ptr(), k_stride, hops.data_ptr(), vis.data_ptr()]
    if fn == "falcon_search":
        rc = lib.falcon_search(*args, _lib.MEM_DEVICE, ctypes.c_void_p(s))
    else:
        rc = lib.falcon_search_noalloc(*args, ctypes.c_void_p(s))
    torch.cuda.synchronize()
    return rc, ids.cpu().numpy(), dists.cpu().numpy(), hops.cpu().numpy(), vis.cpu().numpy()


def _same(a, b):
    return (np.array_equal(a[1], b[1]) and np.array_equal(a[2].view(np.uint32), b[2].view(np.uint32))
            and np.array_equal(a[3], b[3]) and np.array_equal(a[4], b[4]))


@pytest.mark.parametrize("case", ["f32_uniform", "f32_per_query", "bf16_rerank", "intra"])
def test_noalloc_matches_falcon_search_twice(case):
    import torch
    from falcon_b200 import FalconIndex, _lib, make_params
    lib = _lib.load()
    g, q = small_graph("unit", 4000, 96, 64, 80, seed=17)
    ix = FalconIndex(g, storage=("f32", "bf16"))
    dq = torch.from_numpy(q).cuda()
    if case == "f32_per_query":
        rng = np.random.default_rng(3)
        arr = (_lib.SearchParams * len(q))()
        for i in range(len(q)):
            k = int(rng.choice([1, 10, 30]))
            arr[i] = make_params(k=k, ef=int(rng.choice([32, 64, 128])) + k, mc=int(rng.choice([1, 2])),
                                 mg=int(rng.integers(1, 4)))
        params, per_query, ks = arr, True, 30
    elif case == "bf16_rerank":
        params, per_query, ks = make_params(k=10, ef=64, mc=2, mg=2, precision="bf16", rerank=True), False, 10
    elif case == "intra":
        params, per_query, ks = make_params(k=10, ef=64, mc=2, mg=3, mode="intra", channels=4), False, 10
    else:
        params, per_query, ks = make_params(k=10, ef=64, mc=1, mg=4), False, 10
    ref = _reference(lib, ix, q, params, per_query, ks)
    assert ref[0] == _lib.FALCON_OK
    for _ in range(2):
        got = _run(lib, "falcon_search_noalloc", ix, dq, params, per_query, ks)
        assert got[0] == _lib.FALCON_OK, _lib.last_error()
        assert _same(ref, got)
    ix.close()


def test_noalloc_rejects_oversized_and_ef_below_k():
    import torch
    from falcon_b200 import FalconIndex, _lib, make_params
    lib = _lib.load()
    g, q = small_graph("unit", 4000, 96, 64, 8, seed=17)
    ix = FalconIndex(g, storage=("f32", "bf16"))
    big = torch.zeros((3000, 96), dtype=torch.float32, device="cuda")   # 3000 * 256 * 8 B > 4 MiB
    p = make_params(k=10, ef=256, precision="bf16", rerank=True)
    rc = _run(lib, "falcon_search_noalloc", ix, big, p, False, 10)[0]
    assert rc == _lib.FALCON_ERR_ARG
    assert "4 MiB" in _lib.last_error()
    rc = _run(lib, "falcon_search_noalloc", ix, torch.from_numpy(q).cuda(), make_params(k=20, ef=10), False, 20)[0]
    assert rc == _lib.FALCON_ERR_ARG
    # a negative query count and a query stride below the dimension are refused
    # before anything is queued on the stream
    dq = torch.from_numpy(q).cuda()
    out_i = torch.zeros((len(q), 10), dtype=torch.int32, device="cuda")
    out_d = torch.zeros((len(q), 10), dtype=torch.float32, device="cuda")
    p = make_params(k=10, ef=64)
    for nq, stride in ((-1, 96), (len(q), 95)):
        rc = lib.falcon_search_noalloc(ix._h, dq.data_ptr(), nq, stride, None, ctypes.byref(p), 0, out_i.data_ptr(),
                                       out_d.data_ptr(), 10, None, None, None)
        assert rc == _lib.FALCON_ERR_ARG, (nq, stride)
    torch.cuda.synchronize()
    ix.close()
