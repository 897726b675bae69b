"""Known-answer tests of the CPU oracle (no GPU).

The reference ships no tests or golden vectors, so the oracle is pinned by
properties the discretisation must have:
  T2 operator files: field counts, D.1 = 0, D.x = 1;
  T3 free-stream preservation: q = 1, constant velocity => dqdt = 0;
  T4 discrete mass conservation: sum_e sum_n W_n dqdt = 0 (LGL weights);
  T5 spectral accuracy: dqdt -> -u.grad(q) as p grows;
  T9 periodic return: constant velocity with integer displacement returns
     the initial field up to a discretisation error that falls with p;
and GENERAL == OPT1 bit for bit for p <= 7 (same summation order).
"""
import numpy as np
import pytest

import orc
from conftest import rel_maxnorm


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


def lgl_weights(x):
    N = len(x) - 1
    PN = np.polynomial.legendre.legval(x, [0] * N + [1])
    return 2.0 / (N * (N + 1) * PN ** 2)


@pytest.mark.parametrize("p", range(1, 16))
def test_operator_files(p):
    ops = orc.read_operators(p)
    Nq = p + 1
    assert ops.x1D.shape == (Nq,) and ops.Lift_mat.shape == (Nq, Nq, Nq, 6)
    assert ops.x1D[0] == -1.0 and ops.x1D[-1] == 1.0
    assert np.all(np.diff(ops.x1D) > 0)
    assert np.max(np.abs(ops.D1D @ np.ones(Nq))) < 1e-13
    assert np.max(np.abs(ops.D1D @ ops.x1D - 1.0)) < 1e-13
    # token count in the file: Nq + Nq^2 + 6 Nq^3
    with open(f"{orc.OPERATOR_DIR}/p{p}.dat") as f:
        assert len(f.read().split()) == Nq + Nq * Nq + 6 * Nq ** 3


def setup(NeX, NeY, NeZ, p):
    ops = orc.read_operators(p)
    mesh = orc.mesh_setup(NeX, NeY, NeZ, p, ops.x1D)
    return ops, mesh


@pytest.mark.parametrize("p", [1, 3, 7, 8, 15])
def test_free_stream(p):
    ops, mesh = setup(3, 2, 2, p)
    q = np.ones((mesh.Np, mesh.NeA), order="F")
    u = np.full_like(q, 1.0)
    v = np.full_like(q, 0.5)
    w = np.full_like(q, 0.25)
    for ev in (orc.GENERAL, orc.OPT1):
        dq = orc.cal_tend(ev, q, u, v, w, ops, mesh)[:, : mesh.Ne]
        scale = np.max(np.abs(ops.D1D)) * np.max(mesh.Escale)
        assert np.max(np.abs(dq)) < 1e-14 * scale * mesh.Nq


@pytest.mark.parametrize("p", [1, 3, 7, 9, 15])
def test_mass_conservation(p):
    ops, mesh = setup(3, 3, 2, p)
    q, u, v, w = orc.init_fields(mesh, ic_kind=1, seed=7, vel_kind=1)
    W = lgl_weights(ops.x1D)
    Wn = np.einsum("i,j,k->ijk", W, W, W).reshape(-1, order="F")
    for ev in (orc.GENERAL, orc.OPT1):
        dq = orc.cal_tend(ev, q, u, v, w, ops, mesh)[:, : mesh.Ne]
        total = np.sum(Wn[:, None] * dq)
        assert abs(total) < 1e-13 * np.max(np.abs(dq)) * dq.size


def test_spectral_accuracy():
    errs = []
    for p in (1, 3, 5, 7):
        ops, mesh = setup(4, 4, 4, p)
        q, u, v, w = orc.init_fields(mesh, ic_kind=0, vel_kind=0, vel=(1.0, 0.5, 0.25))
        dq = orc.cal_tend(orc.OPT1, q, u, v, w, ops, mesh)[:, : mesh.Ne]
        x, y, z = (mesh.pos_en[:, :, d] for d in range(3))
        tp = 2 * np.pi
        exact = -tp * (1.0 * np.cos(tp * x) * np.sin(tp * y) * np.sin(tp * z)
                       + 0.5 * np.sin(tp * x) * np.cos(tp * y) * np.sin(tp * z)
                       + 0.25 * np.sin(tp * x) * np.sin(tp * y) * np.cos(tp * z))
        errs.append(np.max(np.abs(dq - exact)))
    assert all(b < a for a, b in zip(errs, errs[1:])), errs
    assert errs[-1] < 1e-3


def test_general_equals_opt1_for_low_order():
    for p in (1, 2, 5, 7):
        ops, mesh = setup(2, 3, 2, p)
        q, u, v, w = orc.init_fields(mesh, ic_kind=1, seed=3, vel_kind=1)
        a = orc.cal_tend(orc.GENERAL, q, u, v, w, ops, mesh)
        b = orc.cal_tend(orc.OPT1, q, u, v, w, ops, mesh)
        assert np.array_equal(a, b)


def test_general_and_opt1_differ_only_in_rounding_for_high_order():
    ops, mesh = setup(2, 2, 2, 12)
    q, u, v, w = orc.init_fields(mesh, ic_kind=1, seed=3, vel_kind=1)
    a = orc.cal_tend(orc.GENERAL, q, u, v, w, ops, mesh)
    b = orc.cal_tend(orc.OPT1, q, u, v, w, ops, mesh)
    assert not np.array_equal(a, b)
    assert rel_maxnorm(a, b) < 1e-13


def test_periodic_return():
    errs = []
    for p in (2, 3, 4):
        ops, mesh = setup(4, 4, 4, p)
        q, u, v, w = orc.init_fields(mesh, ic_kind=0, vel_kind=0, vel=(1.0, 0.5, 0.25))
        q_init = q[:, : mesh.Ne].copy()
        h = 0.25
        dt = 0.1 * h / (p + 1) ** 2
        T = 4.0
        nstep = int(round(T / dt))
        orc.run_rk3(orc.OPT1, q, u, v, w, ops, mesh, T / nstep, nstep)
        errs.append(np.max(np.abs(q[:, : mesh.Ne] - q_init)))
    assert all(b < a for a, b in zip(errs, errs[1:])), errs
    assert errs[-1] < 0.05


def test_rk3_reference_run_shape():
    """input.conf of the reference (4^3, p=7, OPT1, dt 1e-3, 1000 steps, print
    every 100) produces ten min/max rows bounded by the sine amplitude."""
    ops, mesh = setup(4, 4, 4, 7)
    q, u, v, w = orc.init_fields(mesh, ic_kind=0)
    diag, times = orc.run_rk3(orc.OPT1, q, u, v, w, ops, mesh, 1.0e-3, 1000, 100)
    assert diag.shape == (10, 3)
    assert np.array_equal(diag[:, 0], np.arange(100, 1001, 100))
    assert np.all(np.abs(diag[:, 1:]) <= 1.0 + 1e-6)
    assert np.all(diag[:, 1] < -0.99) and np.all(diag[:, 2] > 0.99)


@pytest.mark.parametrize("p", [1, 3, 7, 8, 12, 15])
def test_divlike_fields_known_answers(p):
    """divlike_dirXYZ_var5 / gradlike_dirXYZ restated: on LGL nodes the
    derivative matrix differentiates polynomials of degree <= p exactly, so
    f = x^a y^b z^c (a, b, c <= p) has derivatives a x^(a-1) y^b z^c etc.
    Each of nvar fields per element gets its own exponents; GENERAL and OPT1
    agree to rounding (bit for bit for p <= 7)."""
    ops = orc.read_operators(p)
    Nq = p + 1
    x = ops.x1D
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")  # node (i,j,k)
    nvar, Ne = 3, 4
    rng = np.random.default_rng(p)
    ins, want = [], []
    for e in range(Ne):
        for v in range(nvar):
            a_, b_, c_ = rng.integers(0, p + 1, size=3)
            f = X ** a_ * Y ** b_ * Z ** c_
            dx = a_ * X ** max(a_ - 1, 0) * Y ** b_ * Z ** c_
            dy = b_ * X ** a_ * Y ** max(b_ - 1, 0) * Z ** c_
            dz = c_ * X ** a_ * Y ** b_ * Z ** max(c_ - 1, 0)
            # node n = i + Nq*j + Nq^2*k: Fortran order of the (i,j,k) grid
            ins.append(f.ravel(order="F"))
            want.append([d.ravel(order="F") for d in (dx, dy, dz)])
    f = np.concatenate(ins)
    outs = {}
    for ev in (orc.OPT1, orc.GENERAL):
        outs[ev] = orc.divlike_fields(ev, ops.D1D, nvar, Ne, f, f, f)
        for d in range(3):
            ref = np.concatenate([w[d] for w in want])
            assert np.max(np.abs(outs[ev][d] - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))
    for d in range(3):
        if p <= 7:
            assert np.array_equal(outs[orc.OPT1][d], outs[orc.GENERAL][d])
        else:
            assert rel_maxnorm(outs[orc.OPT1][d], outs[orc.GENERAL][d]) < 1e-13
    # separate inputs per direction: out_d depends on in_d only
    zero = np.zeros_like(f)
    ox, oy, oz = orc.divlike_fields(orc.OPT1, ops.D1D, nvar, Ne, f, zero, zero)
    assert np.array_equal(ox, outs[orc.OPT1][0]) and not oy.any() and not oz.any()
