"""Failure detection of the bounded device waits (needs a B200).

The persistent kernel waits on its bulk copies with bounded polls; a wait
that runs out records a timeout in the status word, the block drains its own
copies and returns, and the host turns the status into SDG_ERR_CUDA at the
next synchronising call.  The reference has no device waits (its only error
handling is the file-open check of main.f90:117-122), so these tests cover
this library's own failure path.

The failure is made on the host: a test hook leaves one tile's ring slot
without copies, so nothing is ever in flight for it and the wait ends by its
poll limit; no fault, trap or unbounded wait is involved.
"""
import numpy as np
import pytest

import orc
import sdg_b200 as sdg
from conftest import rel_maxnorm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


def _case(p, dims, seed=3):
    ops = sdg.read_operators(p)
    mesh = sdg.mesh_setup(*dims, p, ops.x1D)
    fields = sdg.init_fields(mesh, ic_kind=1, seed=seed, vel_kind=1)
    return ops, mesh, fields


@pytest.mark.parametrize("flags,p,variant",
                         [(0, 7, sdg.VARIANT_PIPE), (sdg.FLAG_EXACT, 7, sdg.VARIANT_PIPE),
                          (sdg.FLAG_MIXED, 7, sdg.VARIANT_PIPE), (0, 9, sdg.VARIANT_SPLIT),
                          (sdg.FLAG_MIXED, 11, sdg.VARIANT_SPLIT)])
def test_rk_wait_timeout_is_reported_and_handle_recovers(flags, p, variant):
    dims = (4, 4, 4) if p <= 7 else (3, 3, 3)  # 32 tiles of two, or 27 of one
    ops, mesh, (q, u, v, w) = _case(p, dims)
    dt = 0.1 / dims[0] / (p + 1) ** 2
    H = sdg.Handle(ops, mesh, flags)
    H.set_kernel_variant(variant)
    H.set_state(q, u, v, w)
    H.inject_wait_timeout(5, spins=4096)
    H.rk3_steps(dt, 1)               # asynchronous: the error surfaces at sync
    with pytest.raises(sdg.SdgError) as ei:
        H.synchronize()
    assert ei.value.code == sdg.SDG_ERR_CUDA
    assert "timed out" in str(ei.value)
    H.synchronize()                  # the status word was cleared
    # The handle works again once the hook is off.
    H.inject_wait_timeout(-1)
    H.set_state(q, u, v, w)
    H.rk3_steps(dt, 3)
    got = H.get_field()
    H.close()
    H2 = sdg.Handle(ops, mesh, flags)
    H2.set_kernel_variant(sdg.VARIANT_BLOCK)
    H2.set_state(q, u, v, w)
    H2.rk3_steps(dt, 3)
    ref = H2.get_field()
    H2.close()
    assert np.array_equal(got, ref)


def test_tendency_wait_timeout_is_reported():
    """The drop-in tendency call synchronises, so it raises directly."""
    p, dims = 4, (3, 3, 3)
    ops, mesh, (q, u, v, w) = _case(p, dims)
    omesh = orc.mesh_setup(*dims, p, ops.x1D)
    H = sdg.Handle(ops, mesh, sdg.FLAG_EXACT)
    H.set_kernel_variant(sdg.VARIANT_PIPE)
    H.inject_wait_timeout(0, spins=1024)
    with pytest.raises(sdg.SdgError) as ei:
        H.cal_tend(q, u, v, w)
    assert ei.value.code == sdg.SDG_ERR_CUDA
    H.inject_wait_timeout(-1)
    got = H.cal_tend(q, u, v, w)[:, : mesh.Ne]
    ref = orc.cal_tend(orc.OPT1, q, u, v, w, ops, omesh)[:, : mesh.Ne]
    assert np.array_equal(got, ref)
    H.close()


def test_batch_wait_timeout_is_reported_and_batch_recovers():
    ops = {p: sdg.read_operators(p) for p in (3, 5)}
    boxes = [(4, 3, 3, 3), (3, 3, 2, 5), (2, 4, 3, 3)]
    fields = []
    for k, (nx, ny, nz, p) in enumerate(boxes):
        fields.append(sdg.box_fields(nx, ny, nz, p, ops[p].x1D, ic_kind=1, seed=40 + k,
                                     vel_kind=0, vel=tuple(sdg.random_velocity(40 + k))))

    def make():
        b = sdg.Batch(0)
        for (nx, ny, nz, p), f in zip(boxes, fields):
            b.add(nx, ny, nz, p, ops[p], *f, 0.1 / max(nx, ny, nz) / (p + 1) ** 2)
        b.commit(autotune=False)
        return b

    b = make()
    b.inject_wait_timeout(1, spins=2048)
    with pytest.raises(sdg.SdgError) as ei:
        b.run(1)
    assert ei.value.code == sdg.SDG_ERR_CUDA
    assert "timed out" in str(ei.value)
    b.inject_wait_timeout(-1)
    b.run(2)                         # runs clean again (its state is now stale)
    b.close()
    # A fresh batch without the hook matches the single-handle results.
    b = make()
    b.run(2)
    for i, ((nx, ny, nz, p), f) in enumerate(zip(boxes, fields)):
        mesh = sdg.mesh_setup(nx, ny, nz, p, ops[p].x1D)
        H = sdg.Handle(ops[p], mesh, 0)
        n = mesh.Np * mesh.Ne
        full = [np.zeros((mesh.Np, mesh.NeA), order="F") for _ in range(4)]
        for dst, src in zip(full, f):
            dst.reshape(-1, order="F")[:n] = src.reshape(-1, order="F")[:n]
        H.set_state(*full)
        H.rk3_steps(0.1 / max(nx, ny, nz) / (p + 1) ** 2, 2)
        assert np.array_equal(b.get(i), H.get_field()), i
        H.close()
    b.close()
