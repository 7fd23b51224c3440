"""The allocation-free inner product mg_reduce_static, through the C ABI.

It serves callers that cannot allocate device memory (a host engine that owns
all of it, a real-time loop where cudaMalloc/cudaFree would synchronise the
device, code without a solver plan): its scratch is a static array inside the
library.  Its result must equal the plan-based mg_reduce (FP64 sums in a
different block order: 1e-12 relative) on two calls in a row, since the calls
share that array and the second must not see the first one's state.

This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import mg_lib
import mg_scenes
from helpers import gpu_for

pytestmark = pytest.mark.gpu


def _static_reduce(lib, grid_type, a, b, out, stream):
    return lib.mg_reduce_static(ctypes.c_void_p(grid_type.data_ptr()), ctypes.c_void_p(a.data_ptr()),
                                ctypes.c_void_p(b.data_ptr()), ctypes.c_int64(a.numel()),
                                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))


def test_static_reduce_matches_plan_reduce_on_consecutive_calls():
    import torch
    sc = mg_scenes.dam_break_2d(n=128)
    g, _ = gpu_for(sc)
    lib = mg_lib.load()
    rng = np.random.default_rng(21)
    g.p.copy_(torch.from_numpy(rng.standard_normal(sc.res).astype(np.float32)))
    g.Ap.copy_(torch.from_numpy(rng.standard_normal(sc.res).astype(np.float32)))
    g.r[0].copy_(torch.from_numpy(rng.standard_normal(sc.res).astype(np.float32)))
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")

    ref1 = g.reduce(g.p, g.Ap)                       # existing entry point
    assert _static_reduce(lib, g.grid_type[0], g.p, g.Ap, out[0:1], stream) == 0, mg_lib.last_error()
    ref2 = g.reduce(g.r[0], g.r[0])
    assert _static_reduce(lib, g.grid_type[0], g.r[0], g.r[0], out[1:2], stream) == 0, mg_lib.last_error()
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert abs(got[0] - ref1) <= 1e-12 * abs(ref1)
    assert abs(got[1] - ref2) <= 1e-12 * abs(ref2)


def test_static_reduce_rejects_sizes_beyond_its_scratch():
    import torch
    lib = mg_lib.load()
    t = torch.zeros(4, device="cuda")
    lab = torch.zeros(4, dtype=torch.int8, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.mg_reduce_static(ctypes.c_void_p(lab.data_ptr()), ctypes.c_void_p(t.data_ptr()),
                              ctypes.c_void_p(t.data_ptr()), ctypes.c_int64(33_554_433),
                              ctypes.c_void_p(out.data_ptr()), None)
    assert rc == mg_lib.MG_E_TOO_BIG
    assert "static scratch limit" in mg_lib.last_error()


@pytest.mark.parametrize("n", [0, 1, 4097, 256 ** 3, 33_554_432])
def test_static_reduce_sizes(n):
    """No cells (the sum is 0), a ragged count, 4,096 blocks (256^3 cells) and
    the largest count the static scratch holds (8,192 blocks), each twice in a
    row, against an FP64 sum of the same products."""
    import torch
    lib = mg_lib.load()
    g = torch.Generator(device="cuda").manual_seed(n + 7)
    m = max(n, 1)
    a = torch.randn(m, device="cuda", generator=g)
    b = torch.randn(m, device="cuda", generator=g)
    lab = torch.randint(0, 3, (m,), device="cuda", generator=g, dtype=torch.int8)
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    for k in range(2):
        assert lib.mg_reduce_static(ctypes.c_void_p(lab.data_ptr()), ctypes.c_void_p(a.data_ptr()),
                                    ctypes.c_void_p(b.data_ptr()), ctypes.c_int64(n),
                                    ctypes.c_void_p(out[k:k + 1].data_ptr()), ctypes.c_void_p(stream)) == 0, \
            mg_lib.last_error()
    torch.cuda.synchronize()
    fl = (lab[:n] == 0).double()
    ref = float((a[:n].double() * b[:n].double() * fl).sum()) if n else 0.0
    got = out.cpu().numpy()
    for v in got:
        assert abs(v - ref) <= 1e-12 * max(abs(ref), 1.0), (v, ref)
    if n == 0:
        assert got[0] == 0.0 and got[1] == 0.0
