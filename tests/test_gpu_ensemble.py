"""Batched and served ensembles (needs a B200).

T11: each instance's result is the same alone and in the batch / the served
mix: the per-instance arithmetic does not depend on the group, tiling or
kernel variant, so the comparison is bitwise.  The exact batch also equals
the CPU oracle bit for bit.  The server admits requests by device memory
and rejects requests that can never fit.
"""
import time

import numpy as np
import pytest

import orc
import sdg_b200 as sdg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


def instance(p, dims, seed, vel_kind=0):
    ops = sdg.read_operators(p)
    mesh = sdg.mesh_setup(*dims, p, ops.x1D)
    vel = tuple(sdg.random_velocity(seed))
    q, u, v, w = sdg.init_fields(mesh, ic_kind=1, seed=seed, vel_kind=vel_kind, vel=vel)
    dt = 0.1 * (1.0 / max(dims)) / (p + 1) ** 2
    return ops, mesh, (q, u, v, w), dt


def single_run(ops, mesh, fields, dt, nstep, flags):
    h = sdg.Handle(ops, mesh, flags)
    h.set_state(*fields)
    h.rk3_steps(dt, nstep)
    out = h.get_field()
    h.close()
    return out


CASES = [(3, (4, 3, 5), 1), (7, (3, 2, 2), 2), (3, (2, 2, 3), 3), (5, (3, 3, 3), 4),
         (9, (2, 2, 1), 5), (7, (2, 3, 4), 6), (1, (6, 5, 4), 7)]


@pytest.mark.parametrize("flags", [0, sdg.FLAG_MIXED])
def test_batch_equals_single_instances(flags):
    nstep = 6
    b = sdg.Batch(flags)
    insts = [instance(p, dims, seed) for p, dims, seed in CASES]
    ids = [b.add(*dims, p, ops, *fields, dt) for (p, dims, _), (ops, mesh, fields, dt)
           in zip(CASES, insts)]
    b.commit(autotune=True)
    b.run(nstep)
    info = b.info()
    assert info["instances"] == len(CASES)
    assert {g["p"] for g in info["groups"]} == {1, 3, 5, 7, 9}
    for i, (ops, mesh, fields, dt) in zip(ids, insts):
        want = single_run(ops, mesh, fields, dt, nstep, flags)
        assert np.array_equal(b.get(i), want), i
    b.close()


HIGH_CASES = [(8, (2, 3, 2), 11), (9, (2, 2, 3), 12), (10, (2, 2, 2), 13), (11, (3, 2, 2), 14),
              (12, (2, 2, 2), 15), (13, (2, 2, 1), 16), (14, (2, 1, 2), 17)]


@pytest.mark.parametrize("variant", ["split", "pipe", "block"])
@pytest.mark.parametrize("flags", [0, sdg.FLAG_MIXED, sdg.FLAG_EXACT])
def test_forced_batch_variant_equals_single_instances(variant, flags, monkeypatch):
    """SDG_KERNEL forces one kernel variant on every group of a batch whose
    order supports it: the batched split-column kernel (whole-warp parts at
    p = 8, 10-12 and 14, q0 through the ring where the plan holds it, the
    tile context in the slot), the batched pipelined kernel and the
    one-tile-per-block kernel all reproduce the single instances bit for
    bit at p = 8..14, in the fast FP64, mixed and exact forms."""
    monkeypatch.setenv("SDG_KERNEL", variant)
    nstep = 3
    b = sdg.Batch(flags)
    insts = [instance(p, dims, seed) for p, dims, seed in HIGH_CASES]
    ids = [b.add(*dims, p, ops, *fields, dt) for (p, dims, _), (ops, mesh, fields, dt)
           in zip(HIGH_CASES, insts)]
    b.commit(autotune=False)
    b.run(nstep)
    names = {1: "block", 2: "pipe", 3: "blockocc", 4: "split"}
    chosen = {g["p"]: names.get(g["variant"]) for g in b.info()["groups"]}
    if variant in ("pipe", "block"):
        assert all(v == variant for v in chosen.values()), chosen
    else:
        assert sum(v == "split" for v in chosen.values()) >= 5, chosen
    monkeypatch.delenv("SDG_KERNEL")
    for i, (ops, mesh, fields, dt) in zip(ids, insts):
        want = single_run(ops, mesh, fields, dt, nstep, flags)
        assert np.array_equal(b.get(i), want), i
    b.close()


def test_exact_batch_equals_oracle():
    nstep = 4
    b = sdg.Batch(sdg.FLAG_EXACT)
    cases = [(2, (3, 2, 2), 11), (8, (2, 1, 2), 12), (4, (2, 2, 2), 13)]
    insts = [instance(p, dims, seed) for p, dims, seed in cases]
    ids = [b.add(*dims, p, ops, *fields, dt) for (p, dims, _), (ops, mesh, fields, dt)
           in zip(cases, insts)]
    b.commit(autotune=False)
    b.run(nstep)
    for i, (p, dims, _), (ops, mesh, fields, dt) in zip(ids, cases, insts):
        q, u, v, w = (a.copy(order="F") for a in fields)
        om = orc.mesh_setup(*dims, p, ops.x1D)
        orc.run_rk3(orc.OPT1, q, u, v, w, ops, om, dt, nstep)
        assert np.array_equal(b.get(i), q[:, : mesh.Ne]), i
    b.close()


def test_batch_rejects_mismatched_operators():
    b = sdg.Batch(0)
    ops, mesh, fields, dt = instance(3, (2, 2, 2), 1)
    b.add(2, 2, 2, 3, ops, *fields, dt)
    bad = ops._replace(D1D=ops.D1D * 1.0000001)
    with pytest.raises(sdg.SdgError):
        b.add(2, 2, 2, 3, bad, *fields, dt)
    b.close()


def wait_done(srv, ids, timeout=120):
    t0 = time.time()
    while time.time() - t0 < timeout:
        states = [srv.poll(i)[0] for i in ids]
        if all(s in (sdg.SERVE_DONE, sdg.SERVE_FAILED) for s in states):
            return states
        time.sleep(0.01)
    raise TimeoutError("requests did not finish")


def test_served_result_same_alone_and_in_mix():
    p, dims, seed = 5, (3, 4, 2), 21
    ops, mesh, fields, dt = instance(p, dims, seed)
    nstep = 7
    # alone
    srv = sdg.Server()
    rid = srv.submit(*dims, p, ops, *fields, dt, nstep)
    assert wait_done(srv, [rid]) == [sdg.SERVE_DONE]
    alone = srv.result(rid)
    srv.close()
    # in a mix of other orders, sizes and precisions arriving around it
    srv = sdg.Server()
    others = []
    for k, (pp, dd, ss) in enumerate(CASES):
        o_ops, o_mesh, o_fields, o_dt = instance(pp, dd, 100 + ss)
        others.append(srv.submit(*dd, pp, o_ops, *o_fields, o_dt, 3 + 2 * k,
                                 mixed=(k % 2 == 1)))
        if k == 3:
            rid = srv.submit(*dims, p, ops, *fields, dt, nstep)
    states = wait_done(srv, others + [rid])
    assert all(s == sdg.SERVE_DONE for s in states)
    mixed_res = srv.result(rid)
    st = srv.stats()
    assert st["iterations"] >= nstep and st["dof_steps"] > 0
    srv.close()
    assert np.array_equal(alone, mixed_res)
    assert np.array_equal(alone, single_run(ops, mesh, fields, dt, nstep, 0))


def test_server_admits_by_memory_and_rejects_oversize():
    ops, mesh, fields, dt = instance(3, (4, 4, 4), 31)
    per = mesh.Np * mesh.Ne * 8 * 9   # rough device bytes of one FP64 request
    srv = sdg.Server(max_bytes=2.5 * per)
    ids = [srv.submit(4, 4, 4, 3, ops, *fields, dt, 5) for _ in range(6)]
    states = wait_done(srv, ids)
    assert all(s == sdg.SERVE_DONE for s in states)
    waits = [srv.poll(i)[1] for i in ids]
    assert waits[-1] > waits[0]      # later requests queued for memory
    first = srv.result(ids[0])
    for i in ids[1:]:
        assert np.array_equal(srv.result(i), first)
    big_ops, big_mesh, big_fields, big_dt = instance(3, (8, 8, 8), 32)
    with pytest.raises(sdg.SdgError) as e:
        srv.submit(8, 8, 8, 3, big_ops, *big_fields, big_dt, 2)
    assert e.value.code == sdg.SDG_ERR_ARG
    srv.close()
