"""z-slab decomposition over several ranks (CPU, `gloo`).

The box is split into z-slabs, one per rank; after each stage's local
update_halo (mod_mesh.f90:209-221) the ranks exchange their boundary layers
into each other's z halo slots (the halo buffer of mod_mesh.f90:119-130) and
evaluate the tendency of their slab.  The oracle computes every slab's
tendency (OPT1) and the RK stages of main.f90:51-80, so the gathered result
must equal the single-domain oracle run bit for bit.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import orc
from sdg_b200.zslab import ZSlab, slab_range, z_halo_slots


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slab_ranges_cover_the_box():
    for NeZ in (1, 5, 8, 13):
        for R in range(1, NeZ + 1):
            got = [slab_range(NeZ, r, R) for r in range(R)]
            assert got[0][0] == 0 and sum(nz for _, nz in got) == NeZ
            assert all(got[r][0] + got[r][1] == got[r + 1][0] for r in range(R - 1))
            assert max(nz for _, nz in got) - min(nz for _, nz in got) <= 1


def test_single_rank_slots_are_the_periodic_wrap():
    """On one rank the z slots hold, after update_halo, the opposite layer:
    the -z slots the top layer's +z face nodes, in (j, i, fp) order."""
    p, dims = 2, (3, 2, 4)
    ops = orc.read_operators(p)
    m = orc.mesh_setup(*dims, p, ops.x1D)
    lo, hi = z_halo_slots(m.VMapP, m.Np, m.Ne, dims[0], dims[1], dims[2], (p + 1) ** 2)
    Nq, NQ2 = p + 1, (p + 1) ** 2
    src = m.halo_src_map - 1
    k = 0
    for j in range(dims[1]):
        for i in range(dims[0]):
            top = i + dims[0] * (j + dims[1] * (dims[2] - 1))
            bot = i + dims[0] * j
            for fp in range(NQ2):
                assert src[lo[k]] == top * m.Np + NQ2 * (Nq - 1) + fp
                assert src[hi[k]] == bot * m.Np + fp
                k += 1


def _rank_main(rank, world, port, dims, p, nstep, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        ops = orc.read_operators(p)
        gmesh = orc.mesh_setup(*dims, p, ops.x1D)
        gq, gu, gv, gw = orc.init_fields(gmesh, ic_kind=1, seed=9, vel_kind=1)
        sl = ZSlab(*dims, p, ops.x1D, rank, world, orc.mesh_setup)
        m = sl.mesh
        q, u, v, w = (sl.local(a) for a in (gq, gu, gv, gw))

        def halo(f):
            orc.update_halo(f, m)
            flat = f.reshape(-1, order="F")
            sl.exchange(torch.from_numpy(flat), dist,
                        lambda n: torch.empty(n, dtype=torch.float64))

        for f in (u, v, w):
            halo(f)
        dt = 0.1 / max(dims) / (p + 1) ** 2
        ra, rb = (0.0, 0.75, 1.0 / 3.0), (1.0, 0.25, 2.0 / 3.0)
        for _ in range(nstep):
            q0 = q.copy(order="F")
            for s in range(3):
                halo(q)
                dqdt = orc.cal_tend(orc.OPT1, q, u, v, w, ops, m)
                q[:, : m.Ne] = ra[s] * q0[:, : m.Ne] + rb[s] * (q[:, : m.Ne] +
                                                               dt * dqdt[:, : m.Ne])
        out.put((rank, sl.e0, np.ascontiguousarray(q[:, : m.Ne])))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dims,p", [(2, (3, 2, 4), 3), (3, (2, 3, 7), 2),
                                          (2, (2, 2, 2), 5)])
def test_zslab_rk3_equals_single_domain(world, dims, p):
    nstep = 3
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, dims, p, nstep, out))
             for r in range(world)]
    for pr in procs:
        pr.start()
    parts = [out.get(timeout=180) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    ops = orc.read_operators(p)
    gmesh = orc.mesh_setup(*dims, p, ops.x1D)
    q, u, v, w = orc.init_fields(gmesh, ic_kind=1, seed=9, vel_kind=1)
    dt = 0.1 / max(dims) / (p + 1) ** 2
    orc.run_rk3(orc.OPT1, q, u, v, w, ops, gmesh, dt, nstep)
    got = np.zeros((gmesh.Np, gmesh.Ne))
    for rank, e0, part in parts:
        got[:, e0: e0 + part.shape[1]] = part
    assert np.array_equal(got, q[:, : gmesh.Ne])
