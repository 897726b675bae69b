"""The chunked host-buffer calls (needs a B200): sdg_rk3_steps_host equals
sdg_set_field + sdg_rk3_steps + sdg_get_field bit for bit, and sdg_cal_tend
on host arrays equals sdg_cal_tend_dev on the same arrays in device memory.

The call cuts the element range into chunks (runs of z-layers in a box)
and runs the first and last steps chunk by chunk while the state's chunks
go up and come back; every element still sees exactly the kernels of the
resident path, so the state matches to the last bit.  Cases: chunk
boundaries on and off the z-layers, FP64 fast and exact, the mixed form,
one to three steps, the unchunked path of a small mesh, and the handle
still usable afterwards.
"""
import numpy as np
import pytest
import torch

import sdg_b200 as sdg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


def make(dims, p, flags, seed=3):
    ops = sdg.read_operators(p)
    mesh = sdg.mesh_setup(*dims, p, ops.x1D)
    q, u, v, w = sdg.init_fields(mesh, ic_kind=1, seed=seed, vel_kind=1,
                                 vel=(1.0, 0.5, 0.25))
    dt = 0.1 / max(dims) / (p + 1) ** 2
    return ops, mesh, (q, u, v, w), dt


def three_calls(ops, mesh, flags, fields, dt, nsteps):
    h = sdg.Handle(ops, mesh, flags)
    h.set_state(*fields)
    h.rk3_steps(dt, nsteps)
    out = h.get_field()
    h.close()
    return out


def pinned_copy(q, mesh):
    n = mesh.Np * mesh.Ne
    t = torch.empty(n, dtype=torch.float64, pin_memory=True)
    a = t.numpy()
    a[:] = np.asarray(q).reshape(-1, order="F")[:n]
    return t, a


@pytest.mark.parametrize("dims,p,flags,nsteps", [
    ((16, 16, 16), 3, 0, 1),                    # 8 chunks of two z-layers
    ((13, 16, 20), 2, 0, 2),                    # chunk edges inside z-layers
    ((16, 16, 8), 1, sdg.FLAG_EXACT, 3),        # 4 chunks, exact arithmetic
    ((16, 16, 16), 3, sdg.FLAG_MIXED, 2),       # mixed form
    ((12, 12, 16), 7, 0, 1),                    # DMMA lines, two elements a tile
    ((8, 8, 32), 9, 0, 1),                      # split-column kernel
    ((4, 4, 4), 3, 0, 2),                       # too small: the three calls
    ((16, 16, 32), 3, 0, 2),                    # thin end chunks, 16 chunks
    ((16, 16, 32), 2, sdg.FLAG_EXACT, 1),       # the same, exact arithmetic
    ((8, 8, 16), 15, sdg.FLAG_MIXED, 1),        # thin chunks of one z-layer
    ((16, 16, 16), 3, 0, 3),                    # three steps as one plan
    ((16, 16, 32), 3, 0, 5),                    # first and last steps by chunks
])
def test_host_steps_equal_three_calls(dims, p, flags, nsteps):
    ops, mesh, fields, dt = make(dims, p, flags)
    ref = three_calls(ops, mesh, flags, fields, dt, nsteps)
    h = sdg.Handle(ops, mesh, flags)
    for which, a in zip((sdg.FIELD_U, sdg.FIELD_V, sdg.FIELD_W), fields[1:]):
        h.set_field(which, a)
    _keep, qp = pinned_copy(fields[0], mesh)
    h.rk3_steps_host(qp, dt, nsteps)
    got = qp.reshape(mesh.Np, mesh.Ne, order="F")
    assert np.array_equal(got, ref)
    # The handle's resident state is the same state: two more steps on the
    # device agree with two more through the three calls.
    h.rk3_steps(dt, 2)
    more = h.get_field()
    h.close()
    ref2 = three_calls(ops, mesh, flags, (ref,) + tuple(fields[1:]), dt, 2)
    assert np.array_equal(more, ref2)


def test_host_steps_repeat_and_pageable_memory():
    """Repeated calls chain like repeated three-call steps; pageable host
    memory gives the same result (the copies just do not overlap)."""
    ops, mesh, fields, dt = make((16, 16, 16), 2, 0)
    ref = three_calls(ops, mesh, 0, fields, dt, 3)
    h = sdg.Handle(ops, mesh, 0)
    for which, a in zip((sdg.FIELD_U, sdg.FIELD_V, sdg.FIELD_W), fields[1:]):
        h.set_field(which, a)
    q = np.array(fields[0][:, : mesh.Ne], order="F")
    for _ in range(3):
        h.rk3_steps_host(q, dt, 1)
    h.close()
    assert np.array_equal(q, ref)


def test_host_steps_argument_errors():
    ops, mesh, fields, dt = make((16, 16, 8), 1, 0)
    h = sdg.Handle(ops, mesh, 0)
    q = np.array(fields[0][:, : mesh.Ne], order="F")
    with pytest.raises(sdg.SdgError):
        h.rk3_steps_host(q, dt, 1)          # velocities not set
    for which, a in zip((sdg.FIELD_U, sdg.FIELD_V, sdg.FIELD_W), fields[1:]):
        h.set_field(which, a)
    with pytest.raises(sdg.SdgError):
        h.rk3_steps_host(q, dt, -1)
    with pytest.raises(sdg.SdgError):
        h.rk3_steps_host(q[:, :3].copy(order="F"), dt, 1)   # too small
    h.rk3_steps_host(q, dt, 0)              # upload and download only
    assert np.array_equal(q, fields[0][:, : mesh.Ne])
    h.close()


@pytest.mark.parametrize("dims,p,flags", [
    ((16, 16, 8), 1, sdg.FLAG_EXACT),
    ((16, 16, 32), 3, 0),
    ((13, 16, 20), 2, 0),
    ((12, 12, 16), 7, 0),
])
def test_chunked_tendency_call_equals_device_call(dims, p, flags):
    """sdg_cal_tend on host arrays (meshes of 2,048+ elements: the copies
    and the tendency run by element chunks) equals sdg_cal_tend_dev on the
    same arrays in device memory, including a halo buffer that does not
    match the periodic neighbours (both read it where VMapP points)."""
    ops, mesh, fields, dt = make(dims, p, flags)
    q, u, v, w = (np.array(a, order="F") for a in fields)
    halo = slice(mesh.Ne, mesh.NeA)
    q[:, halo] *= 0.5            # a stale halo: the call must still read it
    h = sdg.Handle(ops, mesh, flags)
    got = h.cal_tend(q, u, v, w)[:, : mesh.Ne]
    dev = [torch.from_numpy(a.reshape(-1, order="F")).cuda() for a in (q, u, v, w)]
    out = torch.zeros_like(dev[0])
    h.cal_tend_dev(out, *dev)
    torch.cuda.synchronize()
    ref = out.cpu().numpy().reshape(mesh.Np, mesh.NeA, order="F")[:, : mesh.Ne]
    h.close()
    assert np.array_equal(got, ref)


def test_host_step_graph_follows_array_dt_and_hooks():
    """A one-step call on pinned memory replays a CUDA graph captured for
    that host array and dt: another array, another dt and the wait-timeout
    test hook (whose kernel arguments the graph holds) each take a new
    capture, and every result still equals the three calls."""
    ops, mesh, fields, dt = make((16, 16, 16), 3, 0)
    h = sdg.Handle(ops, mesh, 0)
    h.set_kernel_variant(sdg.VARIANT_PIPE)   # the kernel the hook acts in
    for which, a in zip((sdg.FIELD_U, sdg.FIELD_V, sdg.FIELD_W), fields[1:]):
        h.set_field(which, a)
    _ka, a = pinned_copy(fields[0], mesh)
    _kb, b = pinned_copy(fields[0], mesh)
    h.rk3_steps_host(a, dt, 1)
    h.rk3_steps_host(b, dt, 1)           # another array
    h.rk3_steps_host(a, 0.5 * dt, 1)     # another dt
    h.rk3_steps_host(b, dt, 1)
    one = three_calls(ops, mesh, 0, fields, dt, 1)
    rest = tuple(fields[1:])
    want_a = three_calls(ops, mesh, 0, (one,) + rest, 0.5 * dt, 1)
    want_b = three_calls(ops, mesh, 0, (one,) + rest, dt, 1)
    assert np.array_equal(a.reshape(mesh.Np, mesh.Ne, order="F"), want_a)
    assert np.array_equal(b.reshape(mesh.Np, mesh.Ne, order="F"), want_b)
    # The same array and dt again, now with the hook on: a replay of the
    # old graph would not see it.
    h.inject_wait_timeout(0, spins=1024)
    with pytest.raises(sdg.SdgError) as ei:
        h.rk3_steps_host(a, 0.5 * dt, 1)
    assert ei.value.code == sdg.SDG_ERR_CUDA
    assert "timed out" in str(ei.value)
    h.inject_wait_timeout(-1)
    a[:] = np.asarray(fields[0]).reshape(-1, order="F")[: mesh.Np * mesh.Ne]
    h.rk3_steps_host(a, dt, 1)
    h.close()
    assert np.array_equal(a.reshape(mesh.Np, mesh.Ne, order="F"), one)
