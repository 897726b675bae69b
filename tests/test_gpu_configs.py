"""Parity at the benchmark configurations, after their full step counts
(needs a B200; the oracle runs on all host cores).

C1  8^3 elements, p = 3, GENERAL, constant velocity (1, 0.5, 0.25), seeded
    Gaussian + Fourier initial condition, 100 SSP-RK3 steps: the exact GENERAL
    kernels equal the oracle bit for bit; the fast kernels agree to 1e-12
    relative max-norm.
C2  32^3, p = 7, same velocity and initial condition, 200 steps: fast kernels
    within 1e-12 of the oracle's OPT1 trajectory; the exact OPT1 kernels equal
    it bit for bit.
C3  mixed precision at 32^3 p = 7 and 16^3 p = 15, divergence-free velocity
    (sin 2pi y, sin 2pi z, sin 2pi x), 200 steps, against the oracle's FP64
    OPT1 trajectory: relative L2 <= 1e-5, relative max-norm <= 1e-4, and the
    drift of the FP64 mass diagnostic (LGL weights) <= 1e-6 of the mass.
C4  the 96-instance batched ensemble (Ne per axis U{6..24}, p in {3,5,7,9},
    velocity U[-1,1]^3), 100 steps, FP64 and mixed: sampled instances (the
    two smallest and the median-size one per order) against single-instance
    oracle runs, 1e-12 (FP64) and 1e-5 relative L2 (mixed).

The reference loop these follow is main.f90:51-80 (RK3 coefficients
mod_common.f90:28-30).  Each oracle trajectory is computed once per session.
"""
import functools

import numpy as np
import pytest

import orc
import sdg_b200 as sdg
from conftest import rel_maxnorm
from sdg_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12
MIXED_L2 = 1e-5
MIXED_MAX = 1e-4
MIXED_MASS = 1e-6


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


@functools.lru_cache(maxsize=None)
def _problem(name):
    NeX, NeY, NeZ, p, form, vel, nstep = W.WORKLOADS[name]
    ops = sdg.read_operators(p)
    mesh = sdg.mesh_setup(NeX, NeY, NeZ, p, ops.x1D)
    fields = sdg.init_fields(mesh, **W.fields_kwargs(vel))
    return ops, mesh, fields, W.dt_for(max(NeX, NeY, NeZ), p), nstep


@functools.lru_cache(maxsize=None)
def _oracle(name, evaltype):
    """The oracle's trajectory of workload `name` after its nstep steps,
    and the initial and final FP64 mass."""
    ops, mesh, (q, u, v, w), dt, nstep = _problem(name)
    omesh = orc.mesh_setup(mesh.NeX, mesh.NeY, mesh.NeZ, mesh.p, ops.x1D)
    qo = q.copy(order="F")
    orc.run_rk3(evaltype, qo, u, v, w, ops, omesh, dt, nstep)
    del omesh
    return np.asfortranarray(qo[:, : mesh.Ne])


def _gpu(name, flags, with_mass=False):
    ops, mesh, (q, u, v, w), dt, nstep = _problem(name)
    H = sdg.Handle(ops, mesh, flags)
    H.set_state(q, u, v, w)
    lgl_w = sdg.lgl_weights(ops.x1D)
    jac = 1.0 / (8.0 * mesh.Ne)
    m0 = H.diagnostics(lgl_w, jac)[0] if with_mass else None
    H.rk3_steps(dt, nstep)
    m1 = H.diagnostics(lgl_w, jac)[0] if with_mass else None
    got = H.get_field()
    H.close()
    return got, m0, m1


# ---- C1 -------------------------------------------------------------------
def test_c1_exact_general_bitwise():
    ref = _oracle("fp64_8c_p3", orc.GENERAL)
    got, _, _ = _gpu("fp64_8c_p3", sdg.FLAG_EXACT | sdg.FLAG_ORDER_GENERAL)
    assert np.array_equal(got, ref), rel_maxnorm(got, ref)


def test_c1_fast():
    ref = _oracle("fp64_8c_p3", orc.GENERAL)
    got, _, _ = _gpu("fp64_8c_p3", 0)
    assert rel_maxnorm(got, ref) <= TOL


# ---- C2 -------------------------------------------------------------------
def test_c2_fast_after_200_steps():
    ref = _oracle("fp64_32c_p7", orc.OPT1)
    got, _, _ = _gpu("fp64_32c_p7", 0)
    err = rel_maxnorm(got, ref)
    print(f"C2 fast: rel max-norm {err:.3e} after 200 steps")
    assert err <= TOL


def test_c2_exact_opt1_bitwise_after_200_steps():
    ref = _oracle("fp64_32c_p7", orc.OPT1)
    got, _, _ = _gpu("fp64_32c_p7", sdg.FLAG_EXACT)
    assert np.array_equal(got, ref), rel_maxnorm(got, ref)


# ---- C3 -------------------------------------------------------------------
@pytest.mark.parametrize("name", ["mixed_32c_p7", "mixed_16c_p15"])
def test_c3_mixed_against_oracle(name):
    ref = _oracle(name, orc.OPT1)
    got, m0, m1 = _gpu(name, sdg.FLAG_MIXED, with_mass=True)
    d = got - ref
    l2 = float(np.linalg.norm(d) / np.linalg.norm(ref))
    mx = rel_maxnorm(got, ref)
    drift = abs(m1 - m0) / abs(m0)
    print(f"{name}: rel L2 {l2:.3e}, rel max-norm {mx:.3e}, mass drift {drift:.3e}")
    assert l2 <= MIXED_L2
    assert mx <= MIXED_MAX
    assert drift <= MIXED_MASS


# ---- C4 -------------------------------------------------------------------
def _c4_sample(comp):
    by_p = {}
    for i, it in enumerate(comp):
        by_p.setdefault(it["p"], []).append((it["ne"], i))
    sample = []
    for p, lst in sorted(by_p.items()):
        lst.sort()
        sample += [lst[0][1], lst[1][1], lst[len(lst) // 2][1]]
    return sorted(set(sample))


@functools.lru_cache(maxsize=None)
def _c4_oracle(i):
    it = W.batch_composition()[i]
    ops = orc.read_operators(it["p"])
    om = orc.mesh_setup(it["ne"], it["ne"], it["ne"], it["p"], ops.x1D)
    vel = tuple(orc.random_velocity(it["seed"]))
    q, u, v, w = orc.init_fields(om, ic_kind=1, seed=it["seed"], vel_kind=0, vel=vel)
    orc.run_rk3(orc.OPT1, q, u, v, w, ops, om, it["dt"], 100)
    return np.asfortranarray(q[:, : om.Ne])


@pytest.mark.parametrize("mixed", [False, True])
def test_c4_batched_ensemble_sample_against_oracle(mixed):
    comp = W.batch_composition()
    ops = {p: sdg.read_operators(p) for p in (3, 5, 7, 9)}
    b = sdg.Batch(sdg.FLAG_MIXED if mixed else 0)
    for it in comp:
        vel = tuple(sdg.random_velocity(it["seed"]))
        f = sdg.box_fields(it["ne"], it["ne"], it["ne"], it["p"], ops[it["p"]].x1D,
                           ic_kind=1, seed=it["seed"], vel_kind=0, vel=vel)
        b.add(it["ne"], it["ne"], it["ne"], it["p"], ops[it["p"]], *f, it["dt"])
        del f
    b.commit(autotune=True)
    b.run(100)
    worst = {}
    for i in _c4_sample(comp):
        got = b.get(i)
        ref = _c4_oracle(i)
        if mixed:
            err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
            assert err <= MIXED_L2, (i, comp[i], err)
        else:
            err = rel_maxnorm(got, ref)
            assert err <= TOL, (i, comp[i], err)
        worst[comp[i]["p"]] = max(worst.get(comp[i]["p"], 0.0), err)
    b.close()
    print(f"C4 ({'mixed, rel L2' if mixed else 'FP64, rel max-norm'}) worst per p: {worst}")
