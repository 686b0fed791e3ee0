"""The batched entry point that allocates nothing.

Some callers cannot call cudaMalloc (code that runs inside another
library's memory pool, hosts that reserve the device heap up front, loops
where an allocation could block).  b200qz_solve_batched_noalloc keeps its
batch descriptors in a fixed device array of the library instead.  Its
results must agree with b200qz_solve_batched_dev on the same batch, on
two calls in a row (the second reuses the array the first one filled).
This file is named to be collected last."""
import ctypes

import numpy as np
import pytest

from conftest import EPS

pytestmark = pytest.mark.gpu


def _batch(pkg, torch):
    sizes = [1, 2, 3, 9, 33, 64, 80, 81, 97, 120, 5, 47]
    mats = [pkg.pencils.random_ht(n, 77 * 1000 + i, 0.02) for i, n in enumerate(sizes)]
    b = pkg.Batch(sizes)
    dev = torch.device("cuda:0")
    h0 = torch.from_numpy(b.pack([m[0] for m in mats])).to(dev)
    t0 = torch.from_numpy(b.pack([m[1] for m in mats])).to(dev)
    return b, h0, t0


def _buffers(torch, b, h0, t0):
    h, t = h0.clone(), t0.clone()
    q, z = torch.zeros_like(h), torch.zeros_like(h)
    e = torch.zeros(3 * b.neig, dtype=torch.float64, device=h.device)
    info = torch.full((b.count,), -7, dtype=torch.int32, device=h.device)
    return h, t, q, z, e, info


def _noalloc(pkg, b, h, t, q, z, e, info, stream=None):
    pl = ctypes.POINTER(ctypes.c_longlong)
    pi = ctypes.POINTER(ctypes.c_int)
    vp = ctypes.c_void_p
    return pkg.lib().b200qz_solve_batched_noalloc(
        b.count, b.n.ctypes.data_as(pi), b.moff.ctypes.data_as(pl), b.eoff.ctypes.data_as(pl),
        vp(h.data_ptr()), vp(t.data_ptr()), vp(q.data_ptr()), vp(z.data_ptr()), vp(e.data_ptr()),
        vp(e.data_ptr() + 8 * b.neig), vp(e.data_ptr() + 16 * b.neig), vp(info.data_ptr()), vp(stream))


def test_noalloc_matches_batched_entry(pkg):
    import torch
    b, h0, t0 = _batch(pkg, torch)
    ref = _buffers(torch, b, h0, t0)
    s = pkg.Solver(0)
    try:
        pkg.solve_batched_device(s, b, *(x.data_ptr() for x in ref[:4]), ref[4].data_ptr(),
                                 ref[4].data_ptr() + 8 * b.neig, ref[4].data_ptr() + 16 * b.neig, ref[5].data_ptr())
    finally:
        s.close()
    torch.cuda.synchronize()
    assert (ref[5] == 0).all()
    nrm = max(float(torch.linalg.norm(h0)), float(torch.linalg.norm(t0)))
    tol = 50 * int(b.n.max()) * EPS
    for call in range(2):
        out = _buffers(torch, b, h0, t0)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        stats0 = torch.cuda.memory_stats().get("allocation.all.allocated", 0)
        rc = _noalloc(pkg, b, *out, stream=torch.cuda.current_stream().cuda_stream)
        assert rc == 0, (call, rc)
        torch.cuda.synchronize()
        if call == 1:
            # the call itself took no device memory: neither the driver's free
            # count nor torch's allocator moved (the first call may load the
            # kernel module, so only the second one is checked)
            assert torch.cuda.mem_get_info()[0] == free0
            assert torch.cuda.memory_stats().get("allocation.all.allocated", 0) == stats0
        assert torch.equal(out[5], ref[5]), call
        for a, r in zip(out[:4], ref[:4]):
            assert float(torch.max(torch.abs(a - r))) <= tol * max(1.0, nrm), call
        # eigenvalues: alpha/beta within the same relative tolerance
        ea, er = out[4].cpu().numpy(), ref[4].cpu().numpy()
        assert np.allclose(ea, er, rtol=tol, atol=tol * nrm), call


def test_noalloc_rejects_oversize_batch(pkg):
    import torch
    b = pkg.Batch([4] * 4097)
    dev = torch.device("cuda:0")
    h = torch.zeros(b.elems, dtype=torch.float64, device=dev)
    e = torch.zeros(3 * b.neig, dtype=torch.float64, device=dev)
    info = torch.zeros(b.count, dtype=torch.int32, device=dev)
    assert _noalloc(pkg, b, h, h, h, h, e, info) == -2
