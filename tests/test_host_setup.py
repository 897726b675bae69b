"""The library's host-side set-up against the oracle (no GPU).

T1: VMapM, VMapP and halo_src_map from sdg_mesh_setup are bit-exact with the
restatement of mod_mesh.f90:74-193 (including the serial halo order) for all
p and uneven NeX != NeY != NeZ; the real tables (normals, scale factors, node
positions), the operator reader and the initial-field generators agree bit
for bit too.
"""
import numpy as np
import pytest

import orc
import sdg_b200 as sdg


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


@pytest.mark.parametrize("p", range(1, 16))
def test_operator_reader_matches(p):
    a = sdg.read_operators(p)
    b = orc.read_operators(p)
    for x, y in ((a.x1D, b.x1D), (a.D1D, b.D1D), (a.Lift_mat, b.Lift_mat)):
        assert np.array_equal(x, y)
    assert np.array_equal(sdg.fmask(p), orc.fmask(p))


MESHES = [(1, 1, 1, 1), (2, 3, 4, 1), (3, 2, 5, 2), (4, 4, 4, 3), (5, 3, 2, 4),
          (2, 5, 3, 5), (3, 3, 3, 7), (6, 2, 1, 7), (2, 2, 3, 8), (1, 3, 2, 11),
          (2, 2, 2, 15)]


@pytest.mark.parametrize("NeX,NeY,NeZ,p", MESHES)
def test_mesh_tables_bit_exact(NeX, NeY, NeZ, p):
    x1D = orc.read_operators(p).x1D
    a = sdg.mesh_setup(NeX, NeY, NeZ, p, x1D)
    b = orc.mesh_setup(NeX, NeY, NeZ, p, x1D)
    assert (a.Ne, a.NeA, a.NhaloNode) == (b.Ne, b.NeA, b.NhaloNode)
    for name in ("VMapM", "VMapP", "halo_src_map", "normal_fn", "Escale", "Fscale",
                 "pos_en"):
        x, y = getattr(a, name), getattr(b, name)
        assert x.dtype == y.dtype and x.shape == y.shape, name
        assert np.array_equal(x, y), name


def test_halo_slot_order_is_serial_traversal():
    """Boundary VMapP values count up 1..NhaloNode in (k,j,i,face,node) order."""
    p = 2
    m = sdg.mesh_setup(3, 4, 2, p, orc.read_operators(p).x1D)
    base = m.Np * m.Ne
    vp = m.VMapP.reshape(-1, order="F")
    halo = vp[vp > base] - base
    assert np.array_equal(halo, np.arange(1, m.NhaloNode + 1))


def test_domain_scaling():
    p = 3
    x1D = orc.read_operators(p).x1D
    a = sdg.mesh_setup(3, 2, 4, p, x1D, dom=(2.0, 1.5, 0.5))
    b = orc.mesh_setup(3, 2, 4, p, x1D, dom=(2.0, 1.5, 0.5))
    for name in ("Escale", "Fscale", "pos_en"):
        assert np.array_equal(getattr(a, name), getattr(b, name))


@pytest.mark.parametrize("ic,vk", [(0, 0), (1, 0), (1, 1), (0, 1)])
def test_initial_fields_bit_exact(ic, vk):
    p = 3
    x1D = orc.read_operators(p).x1D
    ma = sdg.mesh_setup(3, 4, 2, p, x1D)
    mb = orc.mesh_setup(3, 4, 2, p, x1D)
    fa = sdg.init_fields(ma, ic_kind=ic, seed=1234, vel_kind=vk, vel=(1.0, 0.5, 0.25))
    fb = orc.init_fields(mb, ic_kind=ic, seed=1234, vel_kind=vk, vel=(1.0, 0.5, 0.25))
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y)


def test_random_velocity():
    for s in (0, 1, 99):
        a, b = sdg.random_velocity(s), orc.random_velocity(s)
        assert np.array_equal(a, b) and np.all(np.abs(a) <= 1.0)


def test_update_halo_host():
    p = 2
    x1D = orc.read_operators(p).x1D
    m = sdg.mesh_setup(2, 3, 2, p, x1D)
    rng = np.random.default_rng(0)
    f = np.asfortranarray(rng.standard_normal((m.Np, m.NeA)))
    g = f.copy(order="F")
    sdg.update_halo(f, m)
    orc.update_halo(g, orc.mesh_setup(2, 3, 2, p, x1D))
    assert np.array_equal(f, g)


@pytest.mark.parametrize("dims,p,vel_kind", [((3, 4, 5), 3, 0), ((2, 3, 2), 9, 1),
                                             ((5, 2, 3), 1, 1), ((1, 1, 1), 15, 0)])
def test_box_fields_equal_init_fields_on_mesh_positions(dims, p, vel_kind):
    """sdg_box_fields forms the node positions where it uses them; the fields
    equal sdg_init_fields on mesh_setup's pos_en bit for bit."""
    ops = sdg.read_operators(p)
    f1 = sdg.box_fields(*dims, p, ops.x1D, ic_kind=1, seed=7, vel_kind=vel_kind,
                        vel=(0.3, -0.2, 0.9))
    m = sdg.mesh_setup(*dims, p, ops.x1D)
    f2 = sdg.init_fields(m, ic_kind=1, seed=7, vel_kind=vel_kind, vel=(0.3, -0.2, 0.9))
    for a, b in zip(f1, f2):
        assert np.array_equal(a, b[:, : m.Ne])
