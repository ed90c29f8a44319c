"""The J entry point that allocates no device memory (rijk_vj_upper_noalloc).

It exists for callers that cannot let a library call cudaMalloc -- programs
whose device memory all belongs to another allocator or to a fixed arena, and
loops where an allocation between Fock builds would synchronise the device.
This test calls it through the C ABI and checks, on two calls in a row, that
it returns what the allocating entry point rijk_vj_upper_dev returns, within
the 1e-10 per-element tolerance of the other J/K tests.  It lives in its own
file, collected last, and must pass alone in a fresh process as well as after
the other tests (the static scratch array keeps the previous call's contents).
"""
import ctypes as C

import numpy as np
import pytest

from rest_b200 import lib
from rest_b200.synth import host_case

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _noalloc(d_tensor, ld, n, naux, d_dm, spin, scale, mode, d_out, stream):
    return lib().rijk_vj_upper_noalloc(C.c_void_p(d_tensor), ld, n, naux, C.c_void_p(d_dm), spin, scale, mode,
                                       C.c_void_p(d_out), C.c_void_p(stream))


@pytest.mark.parametrize("n,naux,spin,mode", [(37, 150, 1, 1), (200, 800, 2, 0), (600, 2400, 1, 1)])
def test_noalloc_matches_allocating_entry_point(ctx, n, naux, spin, mode):
    import torch

    case = host_case(n, naux, max(1, n // 6), seed=77 + n)
    ctx.set_rimatr(case.rimatr, n)
    d_tensor, ld = ctx.tensor_ptr()
    rng = np.random.default_rng(n)
    dms = [case.dm]
    if spin == 2:
        c2 = np.linalg.qr(rng.standard_normal((n, max(1, n // 7))))[0]
        dms.append(c2 @ c2.T)
    dev = torch.device("cuda", torch.cuda.current_device())
    st = ctx.stream
    with torch.cuda.stream(torch.cuda.ExternalStream(st)):
        dm = torch.tensor(np.stack([d.T for d in dms]).ravel(), dtype=torch.float64, device=dev)
        npair = n * (n + 1) // 2
        ref = torch.empty(spin * npair, dtype=torch.float64, device=dev)
        ctx.vj_upper_dev(dm.data_ptr(), spin, 0.75, mode, ref.data_ptr(), st)
        outs = []
        for _ in range(2):  # two calls in a row share the static scratch
            out = torch.full((spin * npair,), float("nan"), dtype=torch.float64, device=dev)
            rc = _noalloc(d_tensor, ld, n, naux, dm.data_ptr(), spin, 0.75, mode, out.data_ptr(), st)
            assert rc == 0
            outs.append(out)
        ctx.synchronize(st)
        torch.cuda.synchronize()
    for out in outs:
        assert torch.isfinite(out).all()
        assert float((out - ref).abs().max()) <= TOL


def test_noalloc_calls_allocate_no_device_memory(ctx):
    """The property the entry point exists for: after the first call (which
    only looks up the array's address), ten more calls leave the device's free
    memory exactly where it was."""
    import torch

    n, naux = 200, 800
    case = host_case(n, naux, 33, seed=5)
    ctx.set_rimatr(case.rimatr, n)
    d_tensor, ld = ctx.tensor_ptr()
    dm = torch.tensor(case.dm.T.ravel(), dtype=torch.float64, device="cuda")
    out = torch.empty(n * (n + 1) // 2, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    assert _noalloc(d_tensor, ld, n, naux, dm.data_ptr(), 1, 1.0, 1, out.data_ptr(), st) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(10):
        assert _noalloc(d_tensor, ld, n, naux, dm.data_ptr(), 1, 1.0, 1, out.data_ptr(), st) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def _tile_stride(n):
    nt = -(-n // 32)
    return nt * (nt + 1) // 2 * 1024


def test_noalloc_rejects_sizes_beyond_its_scratch():
    """Size and stride checks return before any launch, so any non-null
    device pointer serves here (no tensor needs to be loaded)."""
    import torch

    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    d_tensor, ld = x.data_ptr(), _tile_stride(37)
    # n = 2017 at N = 4n needs more than the 32 MiB array (checked before any launch)
    assert _noalloc(d_tensor, _tile_stride(2017), 2017, 4 * 2017, x.data_ptr(), 1, 1.0, 1, x.data_ptr(), 0) == 8
    assert _noalloc(d_tensor, _tile_stride(1409), 1409, 4 * 1409, x.data_ptr(), 2, 1.0, 1, x.data_ptr(), 0) == 8
    # a row stride that does not match the tile-packed layout of the given sizes
    assert _noalloc(d_tensor, ld + 1024, 37, 150, x.data_ptr(), 1, 1.0, 1, x.data_ptr(), 0) == 1
