"""z-slab subdomains on the GPU (needs a B200).

Every slab is a handle with SDG_FLAG_EXTERNAL_HALO: before each RK stage it
updates its own halo (sdg_update_halo_stage), the slabs exchange their
boundary layers into each other's z halo slots, and then each runs the stage
kernel (sdg_rk3_stage), which reads every boundary face from the halo.  Here
all slabs live on one GPU in one process and the exchange is a device copy
between stages (no kernel waits on another); on several GPUs the same blocks
travel by torch.distributed point-to-point operations.  The gathered result
must equal the single-domain handle's bit for bit, in every arithmetic form.
"""
import numpy as np
import pytest
import torch

import orc
import sdg_b200 as sdg
from sdg_b200.zslab import ZSlab, exchange_local

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _build(built):
    return built


@pytest.mark.parametrize("flags", [0, sdg.FLAG_EXACT, sdg.FLAG_MIXED])
@pytest.mark.parametrize("p,dims,R", [(3, (4, 3, 6), 2), (7, (2, 2, 5), 3),
                                      (9, (2, 3, 4), 2)])
def test_slabs_equal_single_domain(p, dims, R, flags):
    nstep = 4
    ops = sdg.read_operators(p)
    gmesh = sdg.mesh_setup(*dims, p, ops.x1D)
    fields = sdg.init_fields(gmesh, ic_kind=1, seed=17, vel_kind=1)
    dt = 0.1 / max(dims) / (p + 1) ** 2

    G = sdg.Handle(ops, gmesh, flags)
    G.set_state(*fields)
    G.rk3_steps(dt, nstep)
    want = G.get_field()
    G.close()

    slabs = [ZSlab(*dims, p, ops.x1D, r, R, sdg.mesh_setup) for r in range(R)]
    hs = []
    for sl in slabs:
        h = sdg.Handle(ops, sl.mesh, flags | sdg.FLAG_EXTERNAL_HALO)
        h.set_state(*(sl.local(f) for f in fields))
        hs.append(h)
    with pytest.raises(sdg.SdgError):
        hs[0].rk3_steps(dt, 1)       # the step needs the caller's exchange

    def sync():
        for h in hs:
            h.synchronize()
        torch.cuda.synchronize()

    sync()
    for which in (sdg.FIELD_U, sdg.FIELD_V, sdg.FIELD_W):
        exchange_local(slabs, [h.resident_array(which) for h in hs])
    for _ in range(nstep):
        for s in (1, 2, 3):
            for h in hs:
                h.update_halo_stage(s)
            sync()
            exchange_local(slabs, [h.stage_input(s) for h in hs])
            torch.cuda.synchronize()
            for h in hs:
                h.rk3_stage(s, dt)
    got = np.zeros_like(want)
    for sl, h in zip(slabs, hs):
        got[:, sl.e0: sl.e0 + sl.mesh.Ne] = h.get_field()
        h.close()
    assert np.array_equal(got, want)
    if flags == sdg.FLAG_EXACT:
        q, u, v, w = (a.copy(order="F") for a in fields)
        om = orc.mesh_setup(*dims, p, ops.x1D)
        orc.run_rk3(orc.OPT1, q, u, v, w, ops, om, dt, nstep)
        assert np.array_equal(got, q[:, : gmesh.Ne])
