"""The allocation-free batched entry point, bosss_b200_batch_evaluate_noalloc.

It exists for callers that cannot call cudaMalloc (a host whose device memory belongs to
another allocator, or a loop that must not synchronise the device with an allocation):
its scratch lives in a fixed array inside the library. This file is collected last, so a
run that stops at the first failure has run every other test before it; it also passes
on its own in a fresh process.

Checked through the C-ABI: two calls in a row give the same results as the allocating
batch entry point (relative L2 <= 1e-12, the tolerance of the parity tests), device free
memory is the same after the first and after the second call (the first call is where the
driver loads the library's module with the array, when no other test did before), and
oversize batches and parts of partitioned grids are rejected. Each round enqueues the
residual and the VJP call on one stream with no synchronisation between them: the call
does not wait for its kernel, and the stream orders the second call's use of the shared
array after the first kernel.
"""
import ctypes

import numpy as np
import pytest

from bosss_b200 import _capi as C
from bosss_b200 import operator as O
from bosss_b200 import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_noalloc_batch_matches_allocating_batch():
    import torch
    probs = P.batched_advection_diffusion(n_instances=9, seed=88, sizes=(3, 4, 5), degrees=(1, 2, 3, 4))
    Uh = np.concatenate([p.U for p in probs])
    Wh = np.random.default_rng(3).uniform(-1, 1, Uh.size)
    with O.BatchEvaluator(probs) as b:
        R_ref = b.evaluate(C.MODE_RESIDUAL, Uh)
        G_ref = b.evaluate(C.MODE_VJP, Uh, Wh)
    evs = [p.evaluator() for p in probs]
    handles = (ctypes.c_void_p * len(evs))(*[e.handle.value for e in evs])
    U = torch.from_numpy(Uh).cuda()
    W = torch.from_numpy(Wh).cuda()
    R = torch.zeros_like(U)
    G = torch.zeros_like(U)
    L = C.lib()
    legacy = ctypes.c_void_p(C.CUDA_STREAM_LEGACY)
    free = []
    try:
        for call in range(2):
            R.fill_(float("nan"))
            G.fill_(float("nan"))
            torch.cuda.synchronize()
            C.check(L.bosss_b200_batch_evaluate_noalloc(len(evs), handles, C.MODE_RESIDUAL, 1.0, 0.0, C.ptr(U), None,
                                                        C.ptr(R), 0.0, legacy))
            C.check(L.bosss_b200_batch_evaluate_noalloc(len(evs), handles, C.MODE_VJP, 1.0, 0.0, C.ptr(U), C.ptr(W),
                                                        C.ptr(G), 0.0, legacy))
            torch.cuda.synchronize()
            free.append(torch.cuda.mem_get_info()[0])
            assert rel(R.cpu().numpy(), R_ref) <= 1e-12, call
            assert rel(G.cpu().numpy(), G_ref) <= 1e-12, call
        assert free[0] == free[1]
        # more instances than the scratch array holds: rejected, nothing launched
        many = (ctypes.c_void_p * 513)(*([evs[0].handle.value] * 513))
        rc = L.bosss_b200_batch_evaluate_noalloc(513, many, C.MODE_RESIDUAL, 1.0, 0.0, C.ptr(U), None, C.ptr(R), 0.0,
                                                 legacy)
        assert rc == C.ERR_BAD_ARG and "512" in C.last_error()
        # a part of a partitioned grid (ghost planes, global box) is rejected, nothing launched
        from bosss_b200 import distributed as Dd
        pr = P.advection_diffusion3d(n=6, k=1, seed=1)
        part = Dd.SlabPartition(pr.grid, 2, 0, pr.dom[0].Np)
        pe = Dd.PartEvaluator(pr.op, pr.grid, [1], [1], part)
        try:
            one = (ctypes.c_void_p * 1)(pe.handle.value)
            rc = L.bosss_b200_batch_evaluate_noalloc(1, one, C.MODE_RESIDUAL, 1.0, 0.0, C.ptr(U), None, C.ptr(R), 0.0,
                                                     legacy)
            assert rc == C.ERR_BAD_ARG and "partitioned" in C.last_error()
        finally:
            pe.Dispose()
    finally:
        for e in evs:
            e.Dispose()
