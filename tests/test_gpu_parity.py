"""GPU parity against the CPU oracle, through the C ABI (needs a B200).

T6  one tendency evaluation, p = 1..15: the fast FMA kernels agree with the
    oracle's OPT1 to <= 1e-12 relative max-norm; the exact kernels equal the
    oracle's OPT1 and GENERAL bit for bit.
    The plus side is read through the caller's halo buffer exactly where
    VMapP points (a stale halo gives the oracle's answer on the same input).
T7  trajectories of the resident RK3 path: <= 1e-12 (fast), bit for bit
    (exact), after many steps.
T10 mixed precision: relative L2 error <= 1e-5 against the FP64 oracle.
Plus the device-pointer entry point, min/max and the FP64 diagnostics.
"""
import numpy as np
import pytest

import orc
import sdg_b200 as sdg
from conftest import rel_maxnorm

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


def dims_for(p):
    return (3, 4, 2) if p <= 5 else ((3, 2, 2) if p <= 9 else (2, 2, 2))


def case(p, dims=None, seed=11, vel_kind=1, ic_kind=1):
    dims = dims or dims_for(p)
    ops = sdg.read_operators(p)
    mesh = sdg.mesh_setup(*dims, p, ops.x1D)
    omesh = orc.mesh_setup(*dims, p, ops.x1D)
    q, u, v, w = sdg.init_fields(mesh, ic_kind=ic_kind, seed=seed, vel_kind=vel_kind,
                                 vel=(1.0, 0.5, 0.25))
    return ops, mesh, omesh, (q, u, v, w)


@pytest.mark.parametrize("p", range(1, 16))
def test_rhs_fast_vs_oracle(p):
    ops, mesh, omesh, (q, u, v, w) = case(p)
    h = sdg.Handle(ops, mesh, 0)
    got = h.cal_tend(q, u, v, w)[:, : mesh.Ne]
    ref = orc.cal_tend(orc.OPT1, q, u, v, w, ops, omesh)[:, : mesh.Ne]
    assert rel_maxnorm(got, ref) <= TOL
    h.close()


@pytest.mark.parametrize("p", range(1, 16))
@pytest.mark.parametrize("order", ["OPT1", "GENERAL"])
def test_rhs_exact_bitwise(p, order):
    ops, mesh, omesh, (q, u, v, w) = case(p)
    flags = sdg.FLAG_EXACT | (sdg.FLAG_ORDER_GENERAL if order == "GENERAL" else 0)
    h = sdg.Handle(ops, mesh, flags)
    got = h.cal_tend(q, u, v, w)[:, : mesh.Ne]
    ev = orc.OPT1 if order == "OPT1" else orc.GENERAL
    ref = orc.cal_tend(ev, q, u, v, w, ops, omesh)[:, : mesh.Ne]
    assert np.array_equal(got, ref), rel_maxnorm(got, ref)
    h.close()


def test_halo_buffer_is_read_through_vmapp():
    """Random values in the halo region (no update_halo): the GPU reads them
    where VMapP points, exactly like the reference."""
    p = 4
    ops, mesh, omesh, (q, u, v, w) = case(p)
    rng = np.random.default_rng(5)
    base = mesh.Np * mesh.Ne
    qf = q.reshape(-1, order="F")
    qf[base: base + mesh.NhaloNode] = rng.standard_normal(mesh.NhaloNode)
    h = sdg.Handle(ops, mesh, sdg.FLAG_EXACT)
    got = h.cal_tend(q, u, v, w)[:, : mesh.Ne]
    ref = orc.cal_tend(orc.OPT1, q, u, v, w, ops, omesh)[:, : mesh.Ne]
    assert np.array_equal(got, ref)
    h.close()


def test_reference_call_surface():
    """advect3d_eq_cal_tend with the reference's argument list."""
    p = 3
    ops, mesh, omesh, (q, u, v, w) = case(p)
    sdg.dg_optr_kernel_setup("OPT1")
    dqdt = np.zeros_like(q)
    m = mesh
    sdg.advect3d_eq_cal_tend(dqdt, q, u, v, w, ops.D1D, ops.D1D_tr, ops.Lift_mat,
                             m.VMapM, m.VMapP, m.normal_fn, m.Escale, m.Fscale,
                             m.Nq, m.Np, m.NfpTot, m.Ne, m.NeA, m.halo_src_map)
    ref = orc.cal_tend(orc.OPT1, q, u, v, w, ops, omesh)
    assert np.array_equal(dqdt[:, : m.Ne], ref[:, : m.Ne])


def run_both(p, dims, nstep, flags, ev=orc.OPT1, vel_kind=1):
    ops, mesh, omesh, (q, u, v, w) = case(p, dims, vel_kind=vel_kind)
    h = 1.0 / max(dims)
    dt = 0.1 * h / (p + 1) ** 2
    H = sdg.Handle(ops, mesh, flags)
    H.set_state(q, u, v, w)
    H.rk3_steps(dt, nstep)
    got = H.get_field()
    qo = q.copy(order="F")
    orc.run_rk3(ev, qo, u, v, w, ops, omesh, dt, nstep)
    H.close()
    return got, qo[:, : mesh.Ne]


@pytest.mark.parametrize("p,dims,nstep", [(1, (4, 3, 2), 40), (3, (4, 4, 3), 30),
                                          (7, (3, 2, 4), 20), (10, (2, 2, 2), 8),
                                          (12, (2, 2, 2), 4), (14, (2, 2, 2), 4)])
def test_trajectory_fast(p, dims, nstep):
    got, ref = run_both(p, dims, nstep, 0)
    assert rel_maxnorm(got, ref) <= TOL


@pytest.mark.parametrize("p,dims,nstep,order",
                         [(2, (3, 4, 2), 25, "OPT1"), (7, (2, 3, 2), 12, "OPT1"),
                          (9, (2, 2, 2), 6, "GENERAL"), (9, (2, 2, 2), 6, "OPT1")])
def test_trajectory_exact_bitwise(p, dims, nstep, order):
    flags = sdg.FLAG_EXACT | (sdg.FLAG_ORDER_GENERAL if order == "GENERAL" else 0)
    ev = orc.GENERAL if order == "GENERAL" else orc.OPT1
    got, ref = run_both(p, dims, nstep, flags, ev)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("p,dims,nstep", [(7, (4, 4, 4), 50), (15, (2, 2, 2), 20)])
def test_mixed_precision_error(p, dims, nstep):
    got, ref = run_both(p, dims, nstep, sdg.FLAG_MIXED)
    err_l2 = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err_l2 <= 1e-5, err_l2
    assert rel_maxnorm(got, ref) <= 1e-4


def test_minmax_and_diagnostics():
    p = 5
    ops, mesh, omesh, (q, u, v, w) = case(p, (3, 3, 3))
    H = sdg.Handle(ops, mesh, 0)
    H.set_state(q, u, v, w)
    mn, mx = H.minmax()
    assert mn == q[:, : mesh.Ne].min() and mx == q[:, : mesh.Ne].max()
    W = sdg.lgl_weights(ops.x1D)
    Wn = np.einsum("i,j,k->ijk", W, W, W).reshape(-1, order="F")
    jac = (1 / 3) ** 3 / 8
    mass, l2 = H.diagnostics(W, jac)
    qe = q[:, : mesh.Ne]
    assert abs(mass - np.sum(Wn[:, None] * jac * qe)) < 1e-13
    assert abs(l2 - np.sqrt(np.sum(Wn[:, None] * jac * qe * qe))) < 1e-13
    # mass is conserved by the scheme to rounding
    dt = 0.1 * (1 / 3) / 36
    H.rk3_steps(dt, 10)
    mass2, _ = H.diagnostics(W, jac)
    assert abs(mass2 - mass) < 1e-13
    H.close()


def test_device_pointer_entry():
    import torch
    p = 6
    ops, mesh, omesh, (q, u, v, w) = case(p)
    H = sdg.Handle(ops, mesh, sdg.FLAG_EXACT)
    dev = [torch.from_numpy(a.reshape(-1, order="F")).cuda() for a in (q, u, v, w)]
    out = torch.zeros_like(dev[0])
    H.cal_tend_dev(out, *dev)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(mesh.Np, mesh.NeA, order="F")[:, : mesh.Ne]
    ref = orc.cal_tend(orc.OPT1, q, u, v, w, ops, omesh)[:, : mesh.Ne]
    assert np.array_equal(got, ref)
    # update_halo on device == host update_halo
    g = dev[0].clone()
    g[mesh.Np * mesh.Ne:] = 0
    H.update_halo_dev(g)
    torch.cuda.synchronize()
    assert np.array_equal(g.cpu().numpy(), q.reshape(-1, order="F"))
    H.close()


def test_full_size_rhs_against_oracle():
    """32^3 elements, p = 7 (16.8 M DOF): one tendency vs the oracle."""
    p = 7
    ops = sdg.read_operators(p)
    mesh = sdg.mesh_setup(32, 32, 32, p, ops.x1D)
    q, u, v, w = sdg.init_fields(mesh, ic_kind=1, seed=1, vel_kind=0, vel=(1.0, 0.5, 0.25))
    H = sdg.Handle(ops, mesh, 0)
    got = H.cal_tend(q, u, v, w)[:, : mesh.Ne]
    H.close()
    omesh = orc.mesh_setup(32, 32, 32, p, ops.x1D)
    ref = orc.cal_tend(orc.OPT1, q, u, v, w, ops, omesh)[:, : mesh.Ne]
    assert rel_maxnorm(got, ref) <= TOL


@pytest.mark.parametrize("variant", [sdg.VARIANT_BLOCK, sdg.VARIANT_PIPE, sdg.VARIANT_SPLIT])
@pytest.mark.parametrize("p", range(1, 16))
def test_kernel_variants_bitwise(p, variant):
    """Both kernel variants (one tile per block; persistent bulk-copy ring)
    reproduce the oracle bit for bit in exact mode, tendency and RK stages."""
    ops, mesh, omesh, (q, u, v, w) = case(p, (3, 2, 3) if p <= 7 else (2, 2, 3))
    h = sdg.Handle(ops, mesh, sdg.FLAG_EXACT)
    h.set_kernel_variant(variant)
    got = h.cal_tend(q, u, v, w)[:, : mesh.Ne]
    ref = orc.cal_tend(orc.OPT1, q, u, v, w, ops, omesh)[:, : mesh.Ne]
    assert np.array_equal(got, ref)
    dt = 0.1 / 3 / (p + 1) ** 2
    h.set_state(q, u, v, w)
    h.rk3_steps(dt, 3)
    got = h.get_field()
    qo = q.copy(order="F")
    orc.run_rk3(orc.OPT1, qo, u, v, w, ops, omesh, dt, 3)
    assert np.array_equal(got, qo[:, : mesh.Ne])
    h.close()


@pytest.mark.parametrize("variant", [sdg.VARIANT_BLOCK, sdg.VARIANT_PIPE, sdg.VARIANT_SPLIT])
@pytest.mark.parametrize("p", [3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15])
def test_mixed_variants_agree(p, variant):
    """Mixed form: the pipelined kernel (packed FP32 line contractions at
    p = 3, 7, 10-15, its own FP32 line layouts at p = 5-7) and the
    one-tile-per-block kernel (scalar lines below p = 13) give the same bits."""
    dims, nstep = ((4, 3, 5) if p <= 7 else (2, 3, 2)), 10
    ops, mesh, omesh, (q, u, v, w) = case(p, dims)
    dt = 0.1 / dims[2] / (p + 1) ** 2
    res = []
    for var in (sdg.VARIANT_BLOCK, variant):
        h = sdg.Handle(ops, mesh, sdg.FLAG_MIXED)
        h.set_kernel_variant(var)
        h.set_state(q, u, v, w)
        h.rk3_steps(dt, nstep)
        res.append(h.get_field())
        h.close()
    assert np.array_equal(res[0], res[1])


def test_partial_last_tile_and_uneven_sizes():
    """Element counts that leave a partial last tile (pipelined variant)."""
    for p, dims in ((2, (5, 3, 1)), (4, (3, 1, 3)), (6, (1, 3, 3)), (7, (3, 3, 1))):
        ops, mesh, omesh, (q, u, v, w) = case(p, dims)
        h = sdg.Handle(ops, mesh, sdg.FLAG_EXACT)
        h.set_kernel_variant(sdg.VARIANT_PIPE)
        got = h.cal_tend(q, u, v, w)[:, : mesh.Ne]
        ref = orc.cal_tend(orc.OPT1, q, u, v, w, ops, omesh)[:, : mesh.Ne]
        assert np.array_equal(got, ref), (p, dims)
        h.close()


@pytest.mark.parametrize("p", [8, 9, 10, 11, 12, 13, 14, 15])
def test_fast_high_order_variants_agree(p):
    """Fast FP64 at p = 8-15: the pipelined kernel (one block per SM from
    p = 11, up to the 227 KB plan of p = 14), the split-column kernel and the
    one-tile-per-block kernel give the same bits over RK steps, and stay
    within 1e-12 of the oracle."""
    dims, nstep = (2, 3, 2), 3
    ops, mesh, omesh, (q, u, v, w) = case(p, dims)
    dt = 0.1 / 3 / (p + 1) ** 2
    res = []
    for var in (sdg.VARIANT_BLOCK, sdg.VARIANT_PIPE, sdg.VARIANT_SPLIT):
        h = sdg.Handle(ops, mesh, 0)
        h.set_kernel_variant(var)
        h.set_state(q, u, v, w)
        h.rk3_steps(dt, nstep)
        res.append(h.get_field())
        h.close()
    assert np.array_equal(res[0], res[1])
    assert np.array_equal(res[0], res[2])
    qo = q.copy(order="F")
    orc.run_rk3(orc.OPT1, qo, u, v, w, ops, omesh, dt, nstep)
    assert rel_maxnorm(res[1], qo[:, : mesh.Ne]) <= TOL


def test_mixed_tensor_core_lines():
    """Kernel variant 5: the mixed form's x/y lines at p = 7 on the tensor
    cores (TF32, three hi/lo passes, TMEM accumulators).  Its rounding
    differs from the FP32 FMA lines, so it is checked against the FP64
    oracle with the mixed form's bar; at other orders the variant falls back
    to the automatic one (same bits)."""
    p, dims, nstep = 7, (4, 4, 4), 50
    ops, mesh, omesh, (q, u, v, w) = case(p, dims)
    dt = 0.1 / 4 / (p + 1) ** 2
    res = {}
    for var in (sdg.VARIANT_AUTO, sdg.VARIANT_TENSOR):
        h = sdg.Handle(ops, mesh, sdg.FLAG_MIXED)
        h.set_kernel_variant(var)
        h.set_state(q, u, v, w)
        h.rk3_steps(dt, nstep)
        res[var] = h.get_field()
        h.close()
    qo = q.copy(order="F")
    orc.run_rk3(orc.OPT1, qo, u, v, w, ops, omesh, dt, nstep)
    ref = qo[:, : mesh.Ne]
    for var, got in res.items():
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= 1e-5, (var, err)
    assert not np.array_equal(res[sdg.VARIANT_AUTO], res[sdg.VARIANT_TENSOR])
    # another order: the variant runs the automatic kernel
    ops, mesh, omesh, (q, u, v, w) = case(5, (3, 3, 2))
    out = []
    for var in (sdg.VARIANT_AUTO, sdg.VARIANT_TENSOR):
        h = sdg.Handle(ops, mesh, sdg.FLAG_MIXED)
        h.set_kernel_variant(var)
        h.set_state(q, u, v, w)
        h.rk3_steps(0.1 / 3 / 36, 5)
        out.append(h.get_field())
        h.close()
    assert np.array_equal(out[0], out[1])
