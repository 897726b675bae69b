"""sdg_minmax_dev_noalloc, the min/max entry point that allocates nothing.

Some callers cannot allocate device memory where they need the diagnostic
(a time loop under a fixed device-memory budget, or code holding only a raw
device array and no handle).  The entry point reduces through a fixed
file-scope device array instead of handle-owned scratch.  This test calls it
through the C ABI and checks it against the existing entry point,
sdg_minmax, on two calls in a row (the second call reuses the scratch the
first one left behind).  It sits in its own file, collected last.
"""
import ctypes

import numpy as np
import pytest

import sdg_b200 as sdg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


def test_noalloc_minmax_matches_sdg_minmax():
    import torch

    p, dims = 5, (4, 3, 5)
    ops = sdg.read_operators(p)
    mesh = sdg.mesh_setup(*dims, p, ops.x1D)
    q, u, v, w = sdg.init_fields(mesh, ic_kind=1, seed=77, vel_kind=1)
    h = sdg.Handle(ops, mesh, 0)
    h.set_state(q, u, v, w)
    n = mesh.Np * mesh.Ne
    q_dev = h.field_dev_ptr(sdg.FIELD_Q)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = h.stream()
    dt = 0.1 / 5 / 36
    for call in range(2):
        want = h.minmax()            # existing entry point (handle scratch)
        rc = sdg.lib().sdg_minmax_dev_noalloc(ctypes.c_void_p(q_dev), n,
                                               ctypes.c_void_p(out.data_ptr()),
                                               ctypes.c_void_p(stream))
        assert rc == sdg.SDG_OK
        h.synchronize()
        got = out.cpu().numpy()
        # Exact for a min/max; the tolerance of the parity tests is 1e-12.
        assert got[0] == want[0] and got[1] == want[1], (call, got, want)
        h.rk3_steps(dt, 3)           # new state for the second call
    h.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    src = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = sdg.lib().sdg_minmax_dev_noalloc(ctypes.c_void_p(src.data_ptr()),
                                           33554432 + 1,
                                           ctypes.c_void_p(out.data_ptr()), None)
    assert rc == sdg.SDG_ERR_ARG
    buf = ctypes.create_string_buffer(512)
    sdg.lib().sdg_last_error(buf, 512)
    assert b"scratch capacity" in buf.value
    # a valid call still works after the rejection
    rc = sdg.lib().sdg_minmax_dev_noalloc(ctypes.c_void_p(src.data_ptr()), 16,
                                           ctypes.c_void_p(out.data_ptr()), None)
    assert rc == sdg.SDG_OK
    torch.cuda.synchronize()
    assert out.cpu().numpy().tolist() == [0.0, 0.0]


@pytest.mark.parametrize("n", [1, 8193, 33554432])
def test_noalloc_sizes_against_torch(n):
    """Edge sizes: one value, a partial second block, and the capacity limit
    (all 4,096 partial slots and the last-block fold), with planted extremes
    in the first and the last block."""
    import torch

    g = torch.Generator(device="cuda").manual_seed(n)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    if n > 1:
        x[n - 1] = 1e6        # maximum in the last (partial) block
        x[3 % n] = -1e6       # minimum in the first block
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    for _ in range(2):        # the second call reuses the shared scratch
        rc = sdg.lib().sdg_minmax_dev_noalloc(ctypes.c_void_p(x.data_ptr()), n,
                                               ctypes.c_void_p(out.data_ptr()), None)
        assert rc == sdg.SDG_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[0] == float(x.min()) and got[1] == float(x.max()), (n, got)
        x.neg_()              # new extremes for the second call
    del x
    torch.cuda.empty_cache()
